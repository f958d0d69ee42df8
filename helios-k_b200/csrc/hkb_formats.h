// hkb_formats.h -- the reference's file formats (host C++).
//
// Inputs: param.dat + command-line overrides (host.h:75-525), the species
// file <path><species>.param (ISO.h:16-219), partition files (host.h:9-73),
// binary line lists (HITRAN 68-byte records host.h:598-649, hitran.cpp:406;
// ExoMol 32-byte records prepareExomol.cpp:222-225).
// Outputs: Out_<name>.dat/.bin, Out_<name>_cbin*.dat, Out_<name>_bin*.dat and
// Info_<name>.dat (heliosk.cu:1837-2462).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace hkb {

struct IsoInfo {
  std::string cid;  // "%3s" of the id (ISO.h:108), matched against records
  double ab = 0.0, Q296 = 0.0, mass = 0.0;
  int g = 0;
  std::string qfile;  // <path><partition file>
};

struct SpeciesInfo {
  int database = 0, id = 0;
  std::string name;
  std::vector<IsoInfo> iso;
  int npfcol = 2, nFiles = 0;
  std::vector<long long> NL;
  std::vector<int> fileLimit;
  std::vector<std::string> dataFilename;  // without the trailing "bin"
  int nStates = 0, ntcol = 0, version = 0;
  double defaultL = 0.0, defaultn = 0.0;
};

// param.dat (define.h:113-161 Param, defaults of heliosk.cu:308-360)
struct Params {
  std::string name;
  double T = 0.0, P = 0.0;
  std::string PFilename = "-", speciesName, SpeciesFilename = "-", ciaSystem = "-";
  std::string path, pathK, bins = "-", edges = "-", subLorentzian = "-";
  double numin = 0.0, numax = 0.0, dnu = 0.0;
  int Nxb = 0, cutMode = 0;
  double cut = 0.0;
  int doResampling = 0, nC = 0, doTransmission = 0, nTr = 0;
  double dTr = 0.0;
  int doStoreFullK = 0, doStoreK = 0, nbins = 0;
  double kmin = 0.0, qalphaL = 0.5, gammaF = 1.0;
  int doMean = 0, units = 0, replaceFiles = 0, profile = 1, doTuning = 1,
      removePlinth = 0, dev = 0, nP = 1;
  std::vector<double> Plist;
};

// Returns 0 or a negative hk_status; msg explains.
int partition_interp(const double *T, const double *Q, int n, double Tq, double *out);
int partition_dlnq(const double *Tq, const double *q, int n, double T, double *out);
int read_q_file(const std::string &fname, int ncol, std::vector<double> &T,
                std::vector<double> &Q, std::string &msg);
int read_species_param(const std::string &path, const std::string &species,
                       SpeciesInfo &sp, std::string &msg);
void line_file_range(const SpeciesInfo &sp, double numin, double numax, int cutMode, double cut,
                     int *fi0, int *fi1);
// One temperature set of a HITRAN-format CIA file (Richard et al. 2012).
struct CiaSet {
  double T = 0.0, numax = 0.0;
  std::vector<double> nu, cia;
};
// The first nsets sets of a CIA file, read as host.h:698-762 reads them
// (fixed-width header fields, then N "nu cia" pairs).
int read_cia_file(const std::string &fname, int nsets, std::vector<CiaSet> &sets, std::string &msg);
// ISO.h:222-277: file name, number of sets and collider mass of a system
bool cia_system(const std::string &system, std::string &file, int *nsets, double *mass1);
int read_sublorentz_file(const std::string &fname, double p[14], std::string &msg);
int read_param_file(const std::string &fname, int argc, char **argv, Params &p,
                    std::string &msg);

}  // namespace hkb
