// edus_run — drop-in replacement of the reference executable (main_MPI.cpp).
//
//   edus_run [input.txt] [workdir] [--device N] [--precision fp64|mixed]
//
// Reads input.txt (default: ./input.txt) exactly as Read_Input does
// (headers/ReadInput.h:332-815), tabulates the model from the files the input
// names relative to workdir (default: the directory of input.txt; the Wannier
// *_tb.dat file is looked up there like the reference's working directory),
// runs the whole time loop of Source_Main/const_dt_evolution.cpp or
// dyn_dt_evolution.cpp on one GPU and writes Output/{EF,J1,J2,Losses,
// TransientAbs}.txt under workdir in the reference's column format
// (Source_Main/open_files.cpp:14-40). The reference's MPI k partition is not
// needed: the whole grid is resident in one device's HBM.
//
// Exit status 0 on success, 1 on any error (the reference exits 1 on a bad
// input), 2 on a usage error.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>

#include "../../include/edus_b200.h"

namespace {

void usage(FILE* f) {
  fprintf(f,
          "usage: edus_run [input.txt] [workdir] [--device N] [--precision fp64|mixed]\n"
          "  runs the time loop of input.txt on one GPU and writes workdir/Output/*.txt\n");
}

int die(const char* what, int rc) {
  fprintf(stderr, "edus_run: %s: %s (%s)\n", what, edus_strerror(rc), edus_last_error());
  return 1;
}

std::string dir_of(const std::string& path) {
  const size_t s = path.find_last_of('/');
  return s == std::string::npos ? std::string(".") : path.substr(0, s ? s : 1);
}

}  // namespace

int main(int argc, char** argv) {
  std::string input, workdir;
  int device = 0, precision = -1;
  for (int i = 1; i < argc; i++) {
    const char* a = argv[i];
    if (!strcmp(a, "-h") || !strcmp(a, "--help")) {
      usage(stdout);
      return 0;
    }
    if (!strcmp(a, "--device") || !strcmp(a, "--precision")) {
      if (i + 1 >= argc) {
        usage(stderr);
        return 2;
      }
      const char* v = argv[++i];
      if (a[2] == 'd') {
        char* end = nullptr;
        device = (int)strtol(v, &end, 10);
        if (!end || *end || device < 0) {
          usage(stderr);
          return 2;
        }
      } else if (!strcmp(v, "fp64")) {
        precision = EDUS_PREC_FP64;
      } else if (!strcmp(v, "mixed")) {
        precision = EDUS_PREC_MIXED;
      } else {
        usage(stderr);
        return 2;
      }
      continue;
    }
    if (a[0] == '-') {
      usage(stderr);
      return 2;
    }
    if (input.empty()) {
      input = a;
    } else if (workdir.empty()) {
      workdir = a;
    } else {
      usage(stderr);
      return 2;
    }
  }
  if (input.empty()) input = "input.txt";
  if (workdir.empty()) workdir = dir_of(input);

  edus_params p;
  int rc = edus_parse_input(input.c_str(), &p);
  if (rc) return die(input.c_str(), rc);
  if (p.coulomb && !p.read_from_files) {
    // the reference computes the Coulomb tables when it does not read them
    // (Source_Main/Fourier_Coulomb.cpp:95-500): generate them on the device
    // into Output/Coulomb and read them back as Read_Coulomb_from_files does
    edus_coulomb_gen_options go;
    edus_coulomb_gen_options_default(&go);
    go.device = device;
    char label[sizeof(p.coulomb_label)];
    int32_t ng = 0;
    rc = edus_coulomb_generate(&p, workdir.c_str(), &go, label, (int32_t)sizeof(label), &ng);
    if (rc) return die("Coulomb coefficients", rc);
    printf("edus_run: Coulomb tables %s (%d G vectors) in %s/Output/Coulomb\n", label, (int)ng, workdir.c_str());
    p.read_from_files = 1;
    snprintf(p.coulomb_label, sizeof(p.coulomb_label), "%s", label);
  }
  edus_problem* pb = nullptr;
  rc = edus_problem_create(&p, workdir.c_str(), &pb);
  if (rc) return die("problem set-up", rc);
  edus_problem_info info;
  edus_problem_info_get(pb, &info);
  edus_problem_write_kpt(pb, workdir.c_str());
  edus_problem_write_test_matrices(pb, workdir.c_str());

  edus_options o;
  edus_options_default(&o);
  o.device = device;
  o.precision = precision;
  edus_ctx* ctx = nullptr;
  rc = edus_create(pb, &o, &ctx);
  if (rc) {
    edus_problem_free(pb);
    return die("device context", rc);
  }
  rc = edus_run(ctx);
  double ms = 0;
  int64_t launches = 0;
  if (!rc) rc = edus_last_timing(ctx, &ms, &launches);
  const std::string out = workdir + "/Output";
  if (!rc) rc = edus_write_outputs(ctx, out.c_str());
  int32_t it = 0, nlog = 0;
  double t = 0, dt = 0;
  if (!rc) rc = edus_clock(ctx, &it, &t, &dt);
  if (!rc) rc = edus_obs_count(ctx, &nlog);
  if (rc) {
    edus_destroy(ctx);
    edus_problem_free(pb);
    return die("time loop", rc);
  }
  printf("edus_run: %d bands, %lld k points, %d steps, %d output instants, %.3f ms on the device (%lld launches)\n",
         (int)info.ncv, (long long)info.nk, (int)it, (int)nlog, ms, (long long)launches);
  printf("edus_run: outputs in %s\n", out.c_str());
  edus_destroy(ctx);
  edus_problem_free(pb);
  return 0;
}
