// heliosk_main.cpp -- drop-in replacement for the reference executable on the
// opacity path.  Same inputs (param.dat + "-flag value" overrides,
// <path><species>.param, partition files, binary line lists) and the same
// outputs (Info_<name>.dat, Out_<name>.dat/.bin, Out_<name>_cbin*.dat,
// Out_<name>_bin*.dat) as heliosk.cu:main, computed through libhkb's C ABI.
//
// Options outside this path (CIA, species mixtures, bins/edges files, unequal
// spacing, sub-Lorentzian, plinth removal, profiles 2-4, transmission and
// means) are rejected with a message instead of being silently ignored.
// Unlike the reference (heliosk.cu:365-367) a failed run exits with status 1.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "hkb.h"
#include "hkb_formats.h"
#include "hkb_types.h"

using namespace hkb;

// Text lines [0, n) formatted by fmt(i, buf, cap) -> length, written to f
// in order.  The formatting (printf %.20g of doubles, the bulk of a
// multi-million-line K file) runs on all host threads in blocks; the bytes
// are those a single fprintf loop writes.
template <class Fmt>
static void write_lines(FILE *f, int64_t n, Fmt fmt) {
  const int64_t block = 1 << 16;
  const int nt = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  std::vector<std::string> out(nt);
  for (int64_t b0 = 0; b0 < n; b0 += block * nt) {
    std::vector<std::thread> th;
    for (int t = 0; t < nt; ++t) {
      th.emplace_back([&, t] {
        std::string &o = out[t];
        o.clear();
        const int64_t a = b0 + t * block, e = std::min(n, a + block);
        char buf[256];
        for (int64_t i = a; i < e; ++i) o.append(buf, (size_t)fmt(i, buf, sizeof buf));
      });
    }
    for (auto &x : th) x.join();
    for (int t = 0; t < nt; ++t) fwrite(out[t].data(), 1, out[t].size(), f);
  }
}

static int die(const std::string &m) {
  printf("%s\n", m.c_str());
  return 1;
}

int main(int argc, char **argv) {
  Params p;
  std::string msg;
  if (read_param_file("param.dat", argc, argv, p, msg) != 0) return die(msg);
  const bool useCia = p.ciaSystem != "-";
  if (useCia && p.SpeciesFilename != "-") return die("Error, not allowed to use a cia system with a molecule");
  // SpeciesFile: "<species> <abundance>" pairs (host.h:463-487, 579-590)
  std::vector<std::string> mixNames;
  std::vector<double> mixAb;
  if (p.SpeciesFilename != "-") {
    FILE *sf = fopen(p.SpeciesFilename.c_str(), "r");
    if (!sf) return die("Error: Species file not found: " + p.SpeciesFilename);
    char b[160];
    double a;
    while (fscanf(sf, "%159s %lf", b, &a) == 2) {
      mixNames.push_back(b);
      mixAb.push_back(a);
    }
    fclose(sf);
    if (mixNames.empty()) return die("Error: no species in file " + p.SpeciesFilename);
  }
  if (p.bins != "-" || p.edges != "-") return die("Error: binsFile / OutputEdgesFile are outside this build's path");
  if (p.Nxb != 0) return die("Error: 'Nnu per bin' (unequal spacing) is outside this build's path");
  double subL[14];
  if (p.subLorentzian != "-" && read_sublorentz_file(p.subLorentzian, subL, msg) != 0) return die(msg);
  if (p.removePlinth != 0 && p.removePlinth != 1) return die("Error: removePlinth must be 0 or 1");
  if (p.profile < 1 || p.profile > 4) return die("Error: profile must be 1, 2, 3 or 4");
  if (p.doTransmission < 0 || p.doTransmission > 2) return die("Error: doTransmission must be 0, 1 or 2");
  if (p.doTransmission > 0 && p.nTr < 1) return die("Error: nTr must be >= 1 for the transmission function");
  if (p.nbins < 1) return die("Error: nbins must be >= 1");

  const char *mode = p.replaceFiles == 0 ? "a" : "w";
  const std::string infoName = "Info_" + p.name + ".dat";
  FILE *info = fopen(infoName.c_str(), mode);
  if (!info) return die("Error: cannot open " + infoName);

  hk_status st;
  hk_ctx *c = hk_create(p.dev, &st);
  if (!c) return die("Error: Device Number is not allowed (hk_create status " + std::to_string(st) + ")");
  auto chk = [&](hk_status s) {
    if (s != HK_OK) {
      printf("Error: %s\n", hk_last_error(c));
      fprintf(info, "Error: %s\n", hk_last_error(c));
      fclose(info);
      hk_destroy(c);
      exit(1);
    }
  };
  cudaEvent_t t0, t1;
  cudaEventCreate(&t0);
  cudaEventCreate(&t1);
  auto seconds = [&]() {
    float ms = 0.f;
    cudaEventSynchronize(t1);
    cudaEventElapsedTime(&ms, t0, t1);
    return ms * 1e-3;
  };

  for (FILE *f : {info, stdout}) {
    fprintf(f, "name = %s\nT = %g\nP = %g\npathToData = %s\nnumin = %g\nnumax = %g\ndnu = %g\n",
            p.name.c_str(), p.T, p.P, p.path.c_str(), p.numin, p.numax, p.dnu);
    fprintf(f, "cutMode = %d\ncut = %g\ndoResampling = %d\nnC = %d\ndoStoreFullK = %d\ndoStoreSK = %d\n",
            p.cutMode, p.cut, p.doResampling, p.nC, p.doStoreFullK, p.doStoreK);
    fprintf(f, "nbins = %d\nkmin = %g\nqalphaL = %g\ngammaF = %g\nUnits = %d\nReplace files = %d\nprofile = %d\n",
            p.nbins, p.kmin, p.qalphaL, p.gammaF, p.units, p.replaceFiles, p.profile);
    if (!mixNames.empty())
      fprintf(f, "Species in file: %s\nNumber of Species: %d\n", p.SpeciesFilename.c_str(), (int)mixNames.size());
    if (p.subLorentzian != "-") fprintf(f, "sub-Lorentzian file: %s\n", p.subLorentzian.c_str());
    if (useCia) fprintf(f, "cia System = %s\n", p.ciaSystem.c_str());
    fprintf(f, "Species Name = %s\nengine = %s\n\n", p.speciesName.c_str(), hk_version());
  }

  chk(hk_set_options(c, p.qalphaL, p.gammaF, p.units, 1.0));
  // mean molar mass over the species (of the mixture), heliosk.cu:665-686;
  // a CIA system's collider mass (heliosk.cu:700-702)
  double meanMass = 0.0;
  if (useCia) {
    chk(hk_load_cia(c, p.path.c_str(), p.ciaSystem.c_str(), &meanMass));
  } else {
    const std::vector<std::string> names = mixNames.empty() ? std::vector<std::string>{p.speciesName} : mixNames;
    for (size_t k = 0; k < names.size(); ++k) {
      SpeciesInfo sp;
      if (read_species_param(p.path, names[k], sp, msg) != 0) return die(msg);
      const double Sscale = names.size() > 1 ? mixAb[k] : 1.0;
      for (auto &iso : sp.iso) meanMass += iso.ab * iso.mass * Sscale;
    }
  }
  double unitScale = 1.0;
  double kmin = p.kmin;
  if (p.units == 1) {  // heliosk.cu:692-701
    unitScale = 1.0 / HK_NA * meanMass;
    kmin /= unitScale;
  }

  const bool compute = p.doStoreFullK >= 0;
  cudaEventRecord(t0);
  if (compute && mixNames.empty() && !useCia)
    chk(hk_load_species_file(c, p.path.c_str(), p.speciesName.c_str(), p.numin, p.numax, p.cutMode, p.cut));
  if (compute && !mixNames.empty()) {
    std::vector<const char *> names;
    for (auto &n : mixNames) names.push_back(n.c_str());
    chk(hk_load_mixture(c, p.path.c_str(), (int)names.size(), names.data(), mixAb.data(), p.numin, p.numax,
                        p.cutMode, p.cut));
  }
  cudaEventRecord(t1);
  const double t_input = compute ? seconds() : 0.0;
  chk(hk_set_grid(c, p.numin, p.numax, p.dnu, p.nbins, p.cutMode, p.cut, kmin));
  chk(hk_set_profile(c, p.profile, p.removePlinth));
  if (p.subLorentzian != "-") chk(hk_set_sublorentzian(c, subL));
  // doTuning = 1: the tile-shape tuner, where its probes pay off (PFile tables)
  chk(hk_set_tuning(c, p.doTuning == 1 ? 1 : 0));
  const int64_t nx = hk_grid_points(c);
  const int nP = p.nP;
  std::vector<double> K((size_t)nP * nx), x(nx);
  for (int64_t i = 0; i < nx; ++i) x[i] = std::fma((double)i, p.dnu, p.numin);  // voigt.h:759
  std::vector<double> Ts(nP, p.T);

  double t_K = 0.0, t_lines = 0.0;
  if (compute) {
    printf("Number of lines: %lld\n", (long long)hk_num_lines(c));
    fprintf(info, "Number of lines: %lld\n", (long long)hk_num_lines(c));
    cudaEventRecord(t0);
    chk(hk_opacity(c, nP, Ts.data(), p.Plist.data(), HK_PRECISION_MIXED, K.data(), 0, nullptr));
    cudaEventRecord(t1);
    // as the reference splits it: K(x) = the line-sum kernels' device time,
    // Lines = the rest of the call (line scaling, first-call workspace, K
    // download)
    const double t_call = seconds();
    double voigt_ms = -1.0;
    hk_last_timing(c, &voigt_ms, nullptr);
    t_K = voigt_ms >= 0.0 ? voigt_ms * 1e-3 : t_call;
    t_lines = t_call - t_K;
    int shape = 0, tuned = -1, ch = 0, gp = 0;
    hk_tuning_result(c, &shape, &tuned, nullptr);
    hk_tile_shape_info(shape, &ch, &gp, nullptr);
    fprintf(info, "Tile shape: %d lines x %d points (%s)\n", ch, gp, tuned >= 0 ? "tuned" : "fixed");
  } else {
    // doStoreFullK = -1 / -2: read K back (heliosk.cu:1860-1935)
    const std::string fn = p.pathK + "Out_" + p.name + (p.doStoreFullK == -1 ? ".dat" : ".bin");
    FILE *f = fopen(fn.c_str(), p.doStoreFullK == -1 ? "r" : "rb");
    if (!f) return die("Error: Input file not found " + fn);
    for (int iP = 0; iP < nP; ++iP) {
      for (int64_t j = 0; j < nx; ++j) {
        if (p.doStoreFullK == -1) {
          double xv, kv, tv, pv;
          int n = (nP == 1) ? fscanf(f, "%lf %lf", &xv, &kv) : fscanf(f, "%lf %lf %lf %lf", &xv, &kv, &tv, &pv);
          if (n < 2) return die("Error: truncated " + fn);
          K[(size_t)iP * nx + j] = kv / unitScale;
        } else {
          float kf;
          if (fread(&kf, sizeof kf, 1, f) != 1) return die("Error: truncated " + fn);
          K[(size_t)iP * nx + j] = (double)kf / unitScale;
        }
      }
    }
    fclose(f);
  }

  // full K output, heliosk.cu:1840-1935
  const auto tw0 = std::chrono::steady_clock::now();
  if (p.doStoreFullK == 1) {
    FILE *f = fopen(("Out_" + p.name + ".dat").c_str(), mode);
    for (int iP = 0; iP < nP; ++iP) {
      const double *Kp = K.data() + (size_t)iP * nx;
      const double Pv = p.Plist[iP];
      write_lines(f, nx, [&](int64_t j, char *buf, size_t cap) {
        if (nP == 1) return snprintf(buf, cap, "%.20g %.20g\n", x[j], Kp[j] * unitScale);
        return snprintf(buf, cap, "%.20g %.20g %.20g %.20g\n", x[j], Kp[j] * unitScale, p.T, Pv);
      });
      fprintf(f, "\n\n");
    }
    fclose(f);
  } else if (p.doStoreFullK == 2) {
    FILE *f = fopen(("Out_" + p.name + ".bin").c_str(), p.replaceFiles == 0 ? "ab" : "wb");
    for (int64_t j = 0; j < (int64_t)nP * nx; ++j) {
      const float kf = (float)(K[j] * unitScale);
      fwrite(&kf, sizeof kf, 1, f);
    }
    fclose(f);
  }

  const double t_write = std::chrono::duration<double>(std::chrono::steady_clock::now() - tw0).count();

  // Planck and Rosseland means, heliosk.cu:1953-2020 (on K in internal units)
  double t_mean = 0.0;
  if (p.doMean > 0) {
    std::vector<double> sums((size_t)nP * 4);
    cudaEventRecord(t0);
    chk(hk_means(c, nP, Ts.data(), K.data(), 0, sums.data(), 0, nullptr));
    cudaEventRecord(t1);
    t_mean = seconds();
    // sigma T^4 / pi and pi / (4 sigma T^3), the reference's analytic integrals
    const double sigma = 2.0 * HK_KB * HK_KB * HK_KB * HK_KB /
                         (HK_H * HK_H * HK_H * HK_C * HK_C * 15.0) * M_PI * M_PI * M_PI * M_PI * M_PI;
    const double integral1 = sigma * p.T * p.T * p.T * p.T / M_PI;
    const double integral2 = M_PI / (4.0 * sigma * p.T * p.T * p.T);
    FILE *f = fopen(("Out_" + p.name + "_mean.dat").c_str(), mode);
    for (int iP = 0; iP < nP; ++iP) {
      const double *m = sums.data() + (size_t)iP * 4;
      if (nP == 1) {
        fprintf(f, "%.20g\n%.20g\n%.20g\n%.20g\n%.20g\n%.20g\n", m[0] / m[2], m[3] / m[1],
                m[2] * p.dnu, integral1, m[3] * p.dnu, 1.0 / integral2);
      } else {
        // the reference prints the last two sums without dnu here
        const double v[6] = {m[0] / m[2], m[3] / m[1], m[2], integral1, m[3], 1.0 / integral2};
        for (double x : v) fprintf(f, "%.20g %.20g %.20g\n", x, p.T, p.Plist[iP]);
      }
    }
    fclose(f);
  }

  // sort + resampling, heliosk.cu:2046-2193
  const int nxb = (int)(nx / p.nbins);
  const bool fit = p.doResampling > 0;
  std::vector<double> coeff, sorted, recon;
  std::vector<int32_t> nxmin;
  double t_fit = 0.0;
  // the transmission function reads the reconstructed (fit) or sorted K
  const bool want_k = p.doStoreK > 0 || p.doTransmission > 0;
  if (fit || want_k) {
    if (fit) {
      coeff.resize((size_t)nP * p.nbins * p.nC);
      nxmin.resize((size_t)nP * p.nbins);
    }
    if (want_k) (fit ? recon : sorted).resize((size_t)nP * nx);
    cudaEventRecord(t0);
    chk(hk_kdist(c, nP, K.data(), 0, p.nC, unitScale, fit ? coeff.data() : nullptr,
                 fit ? nxmin.data() : nullptr, (!fit && want_k) ? sorted.data() : nullptr,
                 (fit && want_k) ? recon.data() : nullptr, 0, nullptr));
    cudaEventRecord(t1);
    t_fit = seconds();
  }
  if (fit) {
    FILE *f = nullptr;
    if (p.doResampling == 1) f = fopen(("Out_" + p.name + "_cbin.dat").c_str(), mode);
    char fn[512];
    if (p.doResampling == 2 && p.replaceFiles == 1)
      for (int i = 0; i < p.nbins; ++i) {
        snprintf(fn, sizeof fn, "Out_%s_cbin%.4d.dat", p.name.c_str(), i);
        fclose(fopen(fn, "w"));
      }
    for (int iP = 0; iP < nP; ++iP) {
      for (int i = 0; i < p.nbins; ++i) {
        if (p.doResampling == 2) {
          snprintf(fn, sizeof fn, "Out_%s_cbin%.4d.dat", p.name.c_str(), i);
          f = fopen(fn, "a");
        }
        const int nm = nxmin[(size_t)iP * p.nbins + i];
        fprintf(f, "%.20g %.20g ", p.kmin, std::fmin(nm / ((double)(nxb - 1)), 1.0));
        for (int ic = 0; ic < p.nC; ++ic) {
          if (nm != nxb) fprintf(f, "%.20g ", coeff[((size_t)iP * p.nbins + i) * p.nC + ic]);
          else fprintf(f, "0.0 ");
        }
        if (nP > 1) fprintf(f, "%.20g %.20g ", p.T, p.Plist[iP]);
        if (p.doResampling == 1) fprintf(f, "\n\n");
        if (p.doResampling == 2) {
          if (i < p.nbins - 1) fprintf(f, "\n");
          fclose(f);
          f = nullptr;
        }
      }
    }
    if (f) fclose(f);
  }
  // per-bin sorted (or reconstructed) K, heliosk.cu:2219-2290
  if (p.doStoreK > 0) {
    const std::vector<double> &Kb = fit ? recon : sorted;
    char fn[512];
    FILE *f = nullptr;
    if (p.doStoreK == 1) f = fopen(("Out_" + p.name + "_bin.dat").c_str(), mode);
    if (p.doStoreK == 2 && p.replaceFiles == 1)
      for (int i = 0; i < p.nbins; ++i) {
        snprintf(fn, sizeof fn, "Out_%s_bin%.4d.dat", p.name.c_str(), i);
        fclose(fopen(fn, "w"));
      }
    for (int iP = 0; iP < nP; ++iP) {
      for (int i = 0; i < p.nbins; ++i) {
        if (p.doStoreK == 2) {
          snprintf(fn, sizeof fn, "Out_%s_bin%.4d.dat", p.name.c_str(), i);
          f = fopen(fn, "a");
        }
        const double *Kp = Kb.data() + (size_t)iP * nx + (size_t)i * nxb;
        const double Pv = p.Plist[iP];
        write_lines(f, nxb, [&](int64_t j, char *buf, size_t cap) {
          const double y = j / ((double)(nxb - 1));
          if (nP == 1) return snprintf(buf, cap, "%g %.20g\n", y, Kp[j] * unitScale);
          return snprintf(buf, cap, "%g %.20g %g %g %d\n", y, Kp[j] * unitScale, p.T, Pv, (int)j);
        });
        if (p.doStoreK == 1) fprintf(f, "\n\n");
        if (p.doStoreK == 2) {
          fclose(f);
          f = nullptr;
        }
      }
    }
    if (f) fclose(f);
  }

  // transmission function, heliosk.cu:2377-2430
  double t_tr = 0.0;
  if (p.doTransmission > 0) {
    const std::vector<double> &Kb = fit ? recon : sorted;
    std::vector<double> Tr((size_t)nP * p.nbins * p.nTr);
    cudaEventRecord(t0);
    chk(hk_transmission(c, nP, Kb.data(), fit ? nxmin.data() : nullptr, 0, p.nTr, p.dTr, Tr.data(), 0,
                        nullptr));
    cudaEventRecord(t1);
    t_tr = seconds();
    char fn[512];
    FILE *f = nullptr;
    if (p.doTransmission == 1) f = fopen(("Out_" + p.name + "_tr.dat").c_str(), mode);
    if (p.doTransmission == 2 && p.replaceFiles == 1)
      for (int i = 0; i < p.nbins; ++i) {
        snprintf(fn, sizeof fn, "Out_%s_tr%.4d.dat", p.name.c_str(), i);
        fclose(fopen(fn, "w"));
      }
    for (int iP = 0; iP < nP; ++iP) {
      for (int i = 0; i < p.nbins; ++i) {
        if (p.doTransmission == 2) {
          snprintf(fn, sizeof fn, "Out_%s_tr%.4d.dat", p.name.c_str(), i);
          f = fopen(fn, "a");
        }
        const double *Tb = Tr.data() + ((size_t)iP * p.nbins + i) * p.nTr;
        const double Pv = p.Plist[iP];
        write_lines(f, p.nTr, [&](int64_t j, char *buf, size_t cap) {
          const double m = exp((double)((int)j - p.nTr / 2) * p.dTr);
          if (nP == 1) return snprintf(buf, cap, "%.20g %.20g\n", m, Tb[j]);
          return snprintf(buf, cap, "%.20g %.20g %.20g %.20g %d\n", m, Tb[j], p.T, Pv, (int)j);
        });
        if (p.doTransmission == 1) fprintf(f, "\n\n");
        if (p.doTransmission == 2) {
          fclose(f);
          f = nullptr;
        }
      }
    }
    if (f) fclose(f);
  }

  for (FILE *f : {info, stdout}) {
    fprintf(f, "Time for input:        %g seconds\n", t_input);
    fprintf(f, "Time for Lines:        %g seconds\n", t_lines);
    fprintf(f, "Time for K(x):         %g seconds\n", t_K);
    fprintf(f, "Time for write K(x):   %g seconds\n", t_write);
    fprintf(f, "Time for sort and Resampling:   %g seconds\n", t_fit);
    if (p.doMean > 0) fprintf(f, "Time for mean K(x):    %g seconds\n", t_mean);
    if (p.doTransmission > 0) fprintf(f, "Time for Transmission:   %g seconds\n", t_tr);
  }
  fclose(info);
  hk_destroy(c);
  return 0;
}
