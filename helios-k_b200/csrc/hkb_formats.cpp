// hkb_formats.cpp -- readers for the reference's input files (host C++).
// Compiled with -ffp-contract=off: the partition interpolation must be the
// same IEEE sequence as the reference's host code.
#include "hkb_formats.h"

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>

#include "hkb.h"

namespace hkb {

// host.h:9-73 (readPartition): walk the (T, Q) table, stop at the first row
// with T1 >= T, interpolate linearly from the previous row.  Returns 1 on
// success, 0 on the reference's error conditions.
int partition_interp(const double *Tq, const double *q, int n, double T, double *out) {
  double T0, T1 = -1.0, q0, q1 = 1.0;
  for (int j = 0; j < 100000; ++j) {
    T0 = T1;
    q0 = q1;
    if (j >= n) return 0;
    T1 = Tq[j];
    q1 = q[j];
    if (T0 == T1 && T0 < T && j > 0) return 0;
    if (T1 > T && j == 0) return 0;
    if (T0 < T && T1 >= T) {
      double tt = (T - T0) / (T1 - T0);
      double qv = (q1 - q0) * tt + q0;
      if (j == 0) qv = q1;
      *out = qv;
      return 1;
    }
  }
  return 0;
}

// d ln Q / dT of the interpolant partition_interp evaluates: the slope of the
// segment holding T over Q(T); at a table node, the mean of the slopes of the
// two segments meeting there (what a central difference sees).
int partition_dlnq(const double *Tq, const double *q, int n, double T, double *out) {
  double Q;
  if (!partition_interp(Tq, q, n, T, &Q) || !(Q > 0.0)) return 0;
  int j = 1;
  while (j < n - 1 && Tq[j] < T) ++j;  // Tq[j-1] < T <= Tq[j] (or the ends)
  if (n < 2) {
    *out = 0.0;
    return 1;
  }
  if (j >= n) j = n - 1;
  double slope = (q[j] - q[j - 1]) / (Tq[j] - Tq[j - 1]);
  if (T == Tq[j] && j + 1 < n) slope = 0.5 * (slope + (q[j + 1] - q[j]) / (Tq[j + 1] - Tq[j]));
  *out = slope / Q;
  return 1;
}

int read_q_file(const std::string &fname, int ncol, std::vector<double> &T,
                std::vector<double> &Q, std::string &msg) {
  FILE *f = fopen(fname.c_str(), "r");
  if (!f) {
    msg = "Error: partition file not found " + fname;
    return HK_ERR_IO;
  }
  if (ncol != 2 && ncol != 3) {
    fclose(f);
    msg = "Error: partition file not specified";
    return HK_ERR_FORMAT;
  }
  T.clear();
  Q.clear();
  double a, b, skip;
  while (true) {
    if (fscanf(f, "%lf", &a) != 1) break;
    if (fscanf(f, "%lf", &b) != 1) break;
    if (ncol == 3 && fscanf(f, "%lf", &skip) != 1) break;
    T.push_back(a);
    Q.push_back(b);
  }
  fclose(f);
  if (T.empty()) {
    msg = "Error: partition function can not be read: " + fname;
    return HK_ERR_FORMAT;
  }
  return 0;
}

// read one "<key> = value" line; returns false if the key does not match
static bool key_line(std::istream &in, const char *key, std::string &rest) {
  std::string line;
  while (std::getline(in, line)) {
    if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
    break;
  }
  size_t k = line.find(key);
  if (k != 0) return false;
  rest = line.substr(strlen(key));
  return true;
}

// ISO.h:16-219 (Init)
int read_species_param(const std::string &path, const std::string &species,
                       SpeciesInfo &sp, std::string &msg) {
  const std::string fname = path + species + ".param";
  std::ifstream in(fname);
  if (!in) {
    msg = "Error, no molecule.param file " + fname;
    return HK_ERR_IO;
  }
  std::string rest;
  auto bad = [&](const char *what) {
    msg = std::string("Error in molecule.param file, ") + what + " (" + fname + ")";
    return HK_ERR_FORMAT;
  };
  if (!key_line(in, "Database =", rest)) return bad("Database");
  sp.database = atoi(rest.c_str());
  if (!key_line(in, "Molecule number =", rest)) return bad("Molecule number");
  sp.id = atoi(rest.c_str());
  if (!key_line(in, "Name =", rest)) return bad("Name");
  {
    std::istringstream ss(rest);
    ss >> sp.name;
  }
  std::string line;
  std::getline(in, line);
  size_t eq = line.find('=');
  if (eq == std::string::npos) return bad("Number of Isotopes");
  std::string k = line.substr(0, eq);
  if (k != "Number of Isotopes " && k != "Number of Isotopologues ") return bad("Number of Isotopes");
  int niso = atoi(line.c_str() + eq + 1);
  if (niso < 1 || niso > 16) return bad("Number of Isotopes (1..16)");
  std::getline(in, line);  // header
  sp.iso.clear();
  for (int i = 0; i < niso; ++i) {
    IsoInfo iso;
    std::string cid, qf;
    if (!(in >> cid >> iso.ab >> iso.Q296 >> iso.g >> iso.mass >> qf)) return bad("isotopologue row");
    char buf[16];
    snprintf(buf, sizeof buf, "%3s", cid.c_str());
    iso.cid = std::string(buf).substr(0, 3);
    iso.qfile = path + qf;
    sp.iso.push_back(iso);
  }
  std::getline(in, line);  // rest of the last row
  if (!key_line(in, "Number of columns in partition File =", rest)) return bad("Number of columns in partition File");
  sp.npfcol = atoi(rest.c_str());
  if (!key_line(in, "Number of line/transition files =", rest)) return bad("Number of line/transition files");
  sp.nFiles = atoi(rest.c_str());
  if (sp.nFiles < 0 || sp.nFiles > 500) return bad("Number of line/transition files (0..500)");
  std::getline(in, line);  // "Number of lines per file :"
  sp.NL.assign(sp.nFiles, 0);
  for (int i = 0; i < sp.nFiles; ++i)
    if (!(in >> sp.NL[i])) return bad("Number of lines per file");
  std::getline(in, line);
  std::getline(in, line);  // "Line file limits :"
  sp.fileLimit.assign(sp.nFiles + 1, 0);
  for (int i = 0; i < sp.nFiles + 1; ++i)
    if (!(in >> sp.fileLimit[i])) return bad("Line file limits");
  std::getline(in, line);
  char buf[1024];
  sp.dataFilename.assign(sp.nFiles, "");
  for (int i = 0; i < sp.nFiles; ++i) {
    const char *p = path.c_str();
    const char *n = sp.name.c_str();
    if (sp.database == 0 || sp.database == 1) {
      if (sp.nFiles > 1) snprintf(buf, sizeof buf, "%s%s_%05d-%05d.", p, n, sp.fileLimit[i], sp.fileLimit[i + 1]);
      else snprintf(buf, sizeof buf, "%s%s.", p, n);
    } else if (sp.database == 2) {
      if (sp.nFiles > 1) snprintf(buf, sizeof buf, "%s%s__%05d-%05d.", p, n, sp.fileLimit[i], sp.fileLimit[i + 1]);
      else snprintf(buf, sizeof buf, "%s%s.", p, n);
    } else {
      msg = "Error: database " + std::to_string(sp.database) +
            " (superlines, Kurucz, NIST, VALD, CDSD) is outside this build's path";
      return HK_ERR_UNSUPPORTED;
    }
    sp.dataFilename[i] = buf;
  }
  std::getline(in, line);  // "#ExoMol :"
  if (!key_line(in, "Number of states =", rest)) return bad("Number of states");
  sp.nStates = atoi(rest.c_str());
  if (!key_line(in, "Number of columns in transition files =", rest)) return bad("Number of columns in transition files");
  sp.ntcol = atoi(rest.c_str());
  if (!key_line(in, "Default value of Lorentzian half-width for all lines =", rest)) return bad("Default value of Lorentzian half-width for all lines");
  sp.defaultL = atof(rest.c_str());
  if (!key_line(in, "Default value of temperature exponent for all lines =", rest)) return bad("Default value of temperature exponent for all lines");
  sp.defaultn = atof(rest.c_str());
  if (!key_line(in, "Version =", rest)) return bad("Version");
  sp.version = atoi(rest.c_str());
  if (sp.database == 1) sp.database = 0;  // HITEMP uses the HITRAN record
  return 0;
}

// heliosk.cu:943-956: the files [fi0, fi1) whose wavenumber range, widened
// by the cut, can reach [numin, numax] (all files for cutMode 1 and 2).
void line_file_range(const SpeciesInfo &sp, double numin, double numax, int cutMode, double cut,
                     int *fi0_out, int *fi1_out) {
  if (cut == 0.0) cut = 1.0e30;
  int fi0 = sp.nFiles, fi1 = 0;
  if (cutMode == 0) {
    for (int fi = 0; fi < sp.nFiles; ++fi) {
      if (sp.fileLimit[fi] - cut <= numax) fi1 = fi + 1;
      else break;
    }
    for (int fi = sp.nFiles - 1; fi >= 0; --fi) {
      if (sp.fileLimit[fi + 1] + cut >= numin) fi0 = fi;
      else break;
    }
  } else {
    fi0 = 0;
    fi1 = sp.nFiles;
  }
  *fi0_out = fi0;
  *fi1_out = fi1;
}

bool cia_system(const std::string &system, std::string &file, int *nsets, double *mass1) {
  struct Sys { const char *name; int nsets; double mass1; };
  // the systems the reference knows, with their set counts and the mass
  // (g/mol) its cm^2/g conversion divides by (ISO.h:226-276)
  static const Sys table[] = {
      {"H2-H2", 113, 2.0 * 1.00794},     {"H2-H2_eq", 10, 2.0 * 1.00794},
      {"H2-H2_norm", 10, 2.0 * 1.00794}, {"H2-He", 339, 4.002602},
      {"H2-He_eq", 10, 4.002602},        {"H2-He_norm", 10, 4.002602},
      {"H2-CH4_eq", 10, 16.04246},       {"H2-CH4_norm", 10, 16.04246},
      {"H2-H", 4, 1.00794}};
  for (const Sys &t : table)
    if (system == t.name) {
      file = system + "_2011.cia";
      *nsets = t.nsets;
      *mass1 = t.mass1;
      return true;
    }
  return false;
}

int read_cia_file(const std::string &fname, int nsets, std::vector<CiaSet> &sets, std::string &msg) {
  FILE *f = fopen(fname.c_str(), "r");
  if (!f) {
    msg = "Error: cia file is not available: " + fname;
    return HK_ERR_IO;
  }
  sets.clear();
  char skip[160], c2[12], c3[9], c4[9];
  for (int it = 0; it < nsets; ++it) {
    CiaSet cs;
    bool good = fgets(skip, 21, f) && fgets(skip, 11, f) && fgets(c2, 11, f) && fgets(c3, 8, f) &&
                fgets(c4, 8, f) && fgets(skip, 11, f) && fgets(skip, 37, f);
    const int n = good ? atoi(c3) : 0;
    if (!good || n < 2) {
      fclose(f);
      msg = "Error: cia file " + fname + ": set " + std::to_string(it) + " is missing or malformed";
      return HK_ERR_FORMAT;
    }
    cs.T = strtod(c4, nullptr);
    cs.numax = strtod(c2, nullptr);
    cs.nu.resize(n);
    cs.cia.resize(n);
    for (int k = 0; k < n; ++k)
      if (fscanf(f, "%lf %lf", &cs.nu[k], &cs.cia[k]) != 2) {
        fclose(f);
        msg = "Error: cia file " + fname + ": set " + std::to_string(it) + " is truncated";
        return HK_ERR_FORMAT;
      }
    if (cs.nu[n - 1] != cs.numax) {
      // host.h:749 ends a set's scan where nu reaches the header's numax
      fclose(f);
      msg = "Error: cia file " + fname + ": set " + std::to_string(it) + " does not end at its numax";
      return HK_ERR_FORMAT;
    }
    for (int k = 1; k < n; ++k)
      if (!(cs.nu[k] > cs.nu[k - 1])) {
        fclose(f);
        msg = "Error: cia file " + fname + ": set " + std::to_string(it) + " is not increasing in nu";
        return HK_ERR_FORMAT;
      }
    if (!fgets(skip, 3, f) && it + 1 < nsets) {
      fclose(f);
      msg = "Error: cia file " + fname + " ends after set " + std::to_string(it);
      return HK_ERR_FORMAT;
    }
    sets.push_back(std::move(cs));
  }
  fclose(f);
  return 0;
}

// host.h:489-515: the sub-Lorentzian file, "name value" for sigma1..3, a
// 4-word header, "name alpha beta epsilon" for B1..B3, a 3-word header and
// the range "lo hi" -> p[14] = {sigma1..3, alpha1, beta1, eps1, ..., lo, hi}
int read_sublorentz_file(const std::string &fname, double p[14], std::string &msg) {
  FILE *f = fopen(fname.c_str(), "r");
  if (!f) {
    msg = "Error: sub-Lorentzian file not found: " + fname;
    return HK_ERR_IO;
  }
  char b[4][160];
  bool good = true;
  for (int k = 0; k < 3 && good; ++k) good = fscanf(f, "%159s %lf", b[0], &p[k]) == 2;
  good = good && fscanf(f, "%159s %159s %159s %159s", b[0], b[1], b[2], b[3]) == 4;
  for (int k = 0; k < 3 && good; ++k)
    good = fscanf(f, "%159s %lf %lf %lf", b[0], &p[3 + 3 * k], &p[4 + 3 * k], &p[5 + 3 * k]) == 4;
  good = good && fscanf(f, "%159s %159s %159s", b[0], b[1], b[2]) == 3;
  good = good && fscanf(f, "%lf %lf", &p[12], &p[13]) == 2;
  fclose(f);
  if (!good) {
    msg = "Error in sub-Lorentzian file read " + fname;
    return HK_ERR_FORMAT;
  }
  return 0;
}

// host.h:75-525 (read_parameters): "key = value" lines, an unknown key is an
// error; then "-flag value" command-line overrides.
int read_param_file(const std::string &fname, int argc, char **argv, Params &p,
                    std::string &msg) {
  FILE *f = fopen(fname.c_str(), "r");
  if (!f) {
    msg = "Error: parameter file not found: " + fname;
    return HK_ERR_IO;
  }
  char line[1024];
  int lineno = 0;
  while (fgets(line, sizeof line, f)) {
    std::string s(line);
    if (s.find_first_not_of(" \t\r\n") == std::string::npos) continue;
    size_t e = s.find_first_of("=:");
    if (e == std::string::npos) {
      msg = "Undefined line in param.dat file: line " + std::to_string(lineno);
      fclose(f);
      return HK_ERR_FORMAT;
    }
    std::string key = s.substr(0, e);
    while (!key.empty() && (key.back() == ' ' || key.back() == '\t')) key.pop_back();
    std::string val = s.substr(e + 1);
    std::istringstream vs(val);
    std::string tok;
    vs >> tok;
    auto D = [&](double &d) { d = atof(tok.c_str()); };
    auto I = [&](int &i) { i = atoi(tok.c_str()); };
    if (key == "name") p.name = tok;
    else if (key == "T") D(p.T);
    else if (key == "P") D(p.P);
    else if (key == "PFile") p.PFilename = tok;
    else if (key == "Species Name") p.speciesName = tok;
    else if (key == "SpeciesFile") p.SpeciesFilename = tok;
    else if (key == "ciaSystem") p.ciaSystem = tok;
    else if (key == "pathToData") p.path = tok;
    else if (key == "numin") D(p.numin);
    else if (key == "numax") D(p.numax);
    else if (key == "dnu") D(p.dnu);
    else if (key == "Nnu per bin") I(p.Nxb);
    else if (key == "cutMode") I(p.cutMode);
    else if (key == "cut") D(p.cut);
    else if (key == "doResampling") I(p.doResampling);
    else if (key == "nC") { I(p.nC); if (p.nC > 100) p.nC = 100; }
    else if (key == "doTransmission") I(p.doTransmission);
    else if (key == "nTr") I(p.nTr);
    else if (key == "dTr") D(p.dTr);
    else if (key == "doStoreFullK") I(p.doStoreFullK);
    else if (key == "pathToK") p.pathK = tok;
    else if (key == "doStoreSK") I(p.doStoreK);
    else if (key == "nbins") I(p.nbins);
    else if (key == "binsFile") p.bins = tok;
    else if (key == "OutputEdgesFile") p.edges = tok;
    else if (key == "kmin") D(p.kmin);
    else if (key == "qalphaL") D(p.qalphaL);
    else if (key == "gammaF") D(p.gammaF);
    else if (key == "doMean") I(p.doMean);
    else if (key == "Units") I(p.units);
    else if (key == "ReplaceFiles") I(p.replaceFiles);
    else if (key == "RLOW") { /* not used anymore, host.h:266-271 */ }
    else if (key == "profile") I(p.profile);
    else if (key == "doTuning") I(p.doTuning);
    else if (key == "removePlinth") I(p.removePlinth);
    else if (key == "subLorentzianfile") p.subLorentzian = tok;
    else {
      msg = "Undefined line in param.dat file: line " + std::to_string(lineno) + " (" + key + ")";
      fclose(f);
      return HK_ERR_FORMAT;
    }
    ++lineno;
  }
  fclose(f);
  // "pathToK =" with an empty value leaves pathK empty (tok == "")
  for (int i = 1; i < argc; i += 2) {
    if (i + 1 >= argc) {
      msg = "Error: Console arguments not valid!";
      return HK_ERR_ARG;
    }
    std::string a = argv[i];
    const char *v = argv[i + 1];
    if (a == "-name") p.name = v;
    else if (a == "-T") p.T = atof(v);
    else if (a == "-P") p.P = atof(v);
    else if (a == "-M") p.speciesName = v;
    else if (a == "-path") p.path = v;
    else if (a == "-pathK") p.pathK = v;
    else if (a == "-numin") p.numin = atof(v);
    else if (a == "-numax") p.numax = atof(v);
    else if (a == "-dnu") p.dnu = atof(v);
    else if (a == "-cutM") p.cutMode = atoi(v);
    else if (a == "-cut") p.cut = atof(v);
    else if (a == "-dR") p.doResampling = atoi(v);
    else if (a == "-nC") p.nC = atoi(v);
    else if (a == "-dT") p.doTransmission = atoi(v);
    else if (a == "-nTr") p.nTr = atoi(v);
    else if (a == "-dTr") p.dTr = atof(v);
    else if (a == "-dSF") p.doStoreFullK = atoi(v);
    else if (a == "-dSS") p.doStoreK = atoi(v);
    else if (a == "-nbins") p.nbins = atoi(v);
    else if (a == "-kmin") p.kmin = atof(v);
    else if (a == "-q") p.qalphaL = atof(v);
    else if (a == "-gammaF") p.gammaF = atof(v);
    else if (a == "-dev") p.dev = atoi(v);
    else if (a == "-Mean") p.doMean = atoi(v);
    else if (a == "-tuning") p.doTuning = atoi(v);
    else {
      msg = "Error: Console arguments not valid!";
      return HK_ERR_ARG;
    }
  }
  if (p.PFilename != "-") {
    FILE *pf = fopen(p.PFilename.c_str(), "r");
    if (!pf) {
      msg = "Error: Pressure file not found: " + p.PFilename;
      return HK_ERR_IO;
    }
    double b;
    p.Plist.clear();
    while (fscanf(pf, "%lf", &b) == 1) p.Plist.push_back(b);
    fclose(pf);
    p.nP = (int)p.Plist.size();
  } else {
    p.Plist.assign(1, p.P);
    p.nP = 1;
  }
  return 0;
}

}  // namespace hkb
