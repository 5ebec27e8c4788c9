// r3d_xrism_cli.cc -- command-line 1D XRISM solve: makes the .xvk table the
// 3D solve reads (solvent_read.cc:10-94) from a solvent deck, on the GPU.
//
//   xrism-b200 deck.xvk -o out.xvk [-T K] [-n ntab] [-r dr] [-c KH|HNC|PSEn]
//              [-t tol] [-m history] [-x mix] [-l ladder] [-s maxstep]
//              [-d device] [-v]
//
// The deck is the header and atom table of an .xvk (any table rows after
// them are ignored); ntab, dr and the temperature come from it unless
// given.  Exit status 0 when the solve converged and the file was written.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/rism3d_b200.h"

static int usage() {
  std::fprintf(stderr,
               "usage: xrism-b200 deck.xvk -o out.xvk [-T K] [-n ntab] [-r dr] "
               "[-c KH|HNC|PSEn] [-t tol] [-m history] [-x mix] [-l ladder] [-s maxstep] "
               "[-d device] [-v]\n");
  return 2;
}

int main(int argc, char **argv) {
  if (argc < 2) return usage();
  const char *deck = nullptr, *out = nullptr;
  r3d_xrism_opts o;
  r3d_xrism_default_opts(&o);
  std::vector<r3d_xrism_atom> atoms(1024);
  int natom = 0;
  // the deck first: its ntab, dr and temperature are the defaults
  for (int i = 1; i < argc; ++i)
    if (argv[i][0] != '-') {
      deck = argv[i];
      break;
    } else if (argv[i][1] != 'v') {
      ++i;
    }
  if (!deck) return usage();
  if (r3d_xrism_read_deck(deck, atoms.data(), (int)atoms.size(), &natom, &o) != R3D_OK) {
    std::fprintf(stderr, "%s\n", r3d_last_error(nullptr));
    return 1;
  }
  for (int i = 1; i < argc; ++i) {
    if (argv[i][0] != '-') continue;
    const char f = argv[i][1];
    if (f == 'v') {
      o.verbose = 1;
      continue;
    }
    if (i + 1 >= argc) return usage();
    const char *v = argv[++i];
    switch (f) {
      case 'o': out = v; break;
      case 'T': o.temperature = std::atof(v); break;
      case 'n': o.ntab = std::atoi(v); break;
      case 'r': o.dr = std::atof(v); break;
      case 't': o.tol = std::atof(v); break;
      case 'm': o.history = std::atoi(v); break;
      case 'x': o.mix = std::atof(v); break;
      case 'l': o.nladder = std::atoi(v); break;
      case 's': o.maxstep = std::atoi(v); break;
      case 'd': o.device = std::atoi(v); break;
      case 'c':
        if (!std::strcmp(v, "KH")) {
          o.closure = R3D_KH;
        } else if (!std::strcmp(v, "HNC")) {
          o.closure = R3D_HNC;
        } else if (!std::strncmp(v, "PSE", 3)) {
          o.closure = R3D_PSE;
          o.pse_n = std::atoi(v + 3 + (v[3] == '-'));
        } else {
          return usage();
        }
        break;
      default: return usage();
    }
  }
  if (!out) return usage();
  std::vector<double> xvv;
  {
    int nv = 0;
    for (int i = 0; i < natom; ++i) nv = std::max(nv, std::abs(atoms[i].sym));
    xvv.assign((size_t)(o.ntab > 0 ? o.ntab : 0) * nv * nv, 0.0);
  }
  r3d_xrism_result r;
  if (r3d_xrism_solve(&o, atoms.data(), natom, xvv.data(), &r) != R3D_OK) {
    std::fprintf(stderr, "%s\n", r3d_last_error(nullptr));
    return 1;
  }
  const char *st = r.status == R3D_CONVERGED ? "converged" : r.status == R3D_DIVERGED ? "diverged" : "maxstep";
  std::printf(" %s after %d evaluations, RMS %.3e, compressibility %.8e 1/Pa, %.1f ms on the GPU\n",
              st, r.steps, r.rms, r.xt, r.ms_device);
  if (r.status != R3D_CONVERGED) return 1;
  if (r3d_xrism_write_xvk(out, &o, atoms.data(), natom, xvv.data(), r.xt) != R3D_OK) {
    std::fprintf(stderr, "%s\n", r3d_last_error(nullptr));
    return 1;
  }
  return 0;
}
