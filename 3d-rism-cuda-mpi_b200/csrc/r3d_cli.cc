// rism3d-b200 -- command-line driver with the reference's flags (main.cu:6-69):
//   -i input.inp  -s structure  -l lambda (LJ sigma scaling, Coulomb off)
//   -e lambda (Coulomb scaling)  -f (no centering)  -z (zero solute charges)
//   -c device
// and extensions: -p fp64|mixed, -m history (history-m Anderson, damping from
// the .inp's m unless -b is given), -b damping, -C KH|HNC|PSEn.
// Runs initialize / iterate / output('m') and writes <stem>.xmu (.xmu0 with -z).
#include <getopt.h>

#include <cstdio>
#include <cstdlib>
#include <cctype>
#include <cstring>
#include <string>

#include "../../include/rism3d_b200.h"

static int die(r3d_ctx *c, const char *what) {
  std::fprintf(stderr, "%s: %s\n", what, r3d_last_error(c));
  return 1;
}

int main(int argc, char **argv) {
  std::string input, structure, closure;
  bool centering = true, q0 = false;
  int device = 0, precision = R3D_FP64, history = 0, adswitch = 0;
  double lambda = 1.0, damping = -1.0;
  int ch;
  while ((ch = getopt(argc, argv, "c:i:s:l:e:fzp:m:b:C:")) != -1) {
    switch (ch) {
      case 'c': device = std::atoi(optarg); break;
      case 'i': input = optarg; break;
      case 's': structure = optarg; break;
      case 'l': lambda = std::atof(optarg); adswitch = 1; break;
      case 'e': lambda = std::atof(optarg); adswitch = 2; break;
      case 'f': centering = false; break;
      case 'z': q0 = true; break;
      case 'p': precision = std::strcmp(optarg, "mixed") == 0 ? R3D_MIXED : R3D_FP64; break;
      case 'm': history = std::atoi(optarg); break;
      case 'b': damping = std::atof(optarg); break;
      case 'C': closure = optarg; break;
      default: return 2;
    }
  }
  if (input.empty()) {
    if (optind >= argc) {
      std::printf("No input file!\n");
      return 1;
    }
    input = argv[optind];
  }
  r3d_opts o{};
  o.device = device;
  o.precision = precision;
  o.verbose = 1;
  r3d_ctx *c = nullptr;
  if (r3d_create(&o, &c)) return die(nullptr, "create");
  if (adswitch && r3d_set_ad(c, lambda, adswitch)) return die(c, "set_ad");
  std::printf("reading input data file  : %s\n", input.c_str());
  if (r3d_load_inp(c, input.c_str(), structure.empty() ? nullptr : structure.c_str(),
                   centering, q0))
    return die(c, "input");
  if (r3d_load_xvk(c, nullptr)) return die(c, "solvent");
  if (!closure.empty()) {
    int cl = closure == "HNC" ? R3D_HNC : closure == "KH" ? R3D_KH : R3D_PSE;
    int n = cl == R3D_PSE ? std::atoi(closure.c_str() + 3 + (closure[3] == '-')) : 1;
    if (r3d_set_closure(c, cl, n)) return die(c, "closure");
  }
  if (history > 0 && r3d_set_mixer(c, R3D_MIX_ANM, history, damping)) return die(c, "mixer");
  if (r3d_initialize(c)) return die(c, "initialize");
  // iterate.cu:26-35: a saved <stem>.tuv is the starting t
  const std::string stem = input.substr(0, input.rfind('.'));
  if (FILE *tf = std::fopen((stem + ".tuv").c_str(), "r")) {
    std::fclose(tf);
    std::printf("restarting from %s.tuv\n", stem.c_str());
    if (r3d_read_tuv(c, (stem + ".tuv").c_str())) return die(c, "read_tuv");
  }
  int steps = 0, status = 0;
  double rms = 0;
  if (r3d_iterate(c, &steps, &rms, &status)) return die(c, "iterate");
  double ms = 0;
  r3d_iter_timing(c, &ms, nullptr);
  std::printf("Iteration   :\t%lf sec. (%d steps, %.3f ms/step)\n", ms * steps * 1e-3, steps, ms);
  if (status != R3D_DIVERGED) {
    // output.cu: the files of the deck's outlist
    if (r3d_output(c, nullptr)) return die(c, "output");
  }
  r3d_destroy(c);
  return status == R3D_DIVERGED ? 3 : 0;
}
