// CHECKER — test infrastructure, not product code.
// Runs ONE participant of the reference's own decentralized SVD
// (Excalibur DecentralizedClient, client.cpp:130-208 and run() :447-1310)
// over loopback TCP, exactly as its main.cpp would, then writes the
// participant's outputs as raw float64 files:
//   <out>/sigma.bin   singular values (recomputed from the participant's
//                     final bidiagonal with the reference's own bisection,
//                     the same call run() makes at client.cpp:984)
//   <out>/U.bin       FinalU (client 0 only): m x sigma_count row-major, or
//                     sigma_count x m when m > global_n (client.cpp:1071-1105)
//   <out>/VT.bin      FinalVT, sigma_count x local_n row-major
//   <out>/w.bin       w_lr, local_n (svd_mode 4, linear regression)
//   <out>/ab.bin      alpha[k], beta[k-1] after the lower->upper rotation,
//                     k = min(m, global_n) (the bidiagonal's order, :805-814)
//   <out>/time.txt    the reference's own run() timer (run_begin..run_finish)
//                     followed by its phase timers
// Usage: ref_pipeline cid nclient m local_n port dpath logdir seed mode topk out [opt_control]
// (opt_control defaults to 3, the masks run() applies with block_shift_mask;
// 0 and 2 select the dense block_mask, client.cpp:549-555, 598-601)
#include <algorithm>
#include <cstdio>
#include <string>
#include <unistd.h>
#include "client.hpp"

static void dump(const std::string& f, const double* p, size_t n) {
  FILE* fp = fopen(f.c_str(), "wb");
  if (!fp) { perror(f.c_str()); _exit(3); }
  fwrite(p, sizeof(double), n, fp);
  fclose(fp);
}

int main(int argc, char** argv) {
  if (argc < 12) { fprintf(stderr, "usage: see source\n"); return 2; }
  int cid = atoi(argv[1]), nc = atoi(argv[2]);
  size_t m = strtoull(argv[3], 0, 10), ln = strtoull(argv[4], 0, 10);
  int port = atoi(argv[5]);
  std::string dpath = argv[6], logdir = argv[7];
  unsigned seed = (unsigned)strtoul(argv[8], 0, 10);
  int mode = atoi(argv[9]);
  int topk = atoi(argv[10]);
  std::string out = argv[11];
  const int opt = argc > 12 ? atoi(argv[12]) : 3;
  mkl_set_num_threads(omp_get_max_threads());
  omp_set_num_threads(omp_get_max_threads());
  DecentralizedClient* c = new DecentralizedClient(cid, nc, mode, (size_t)topk, m, ln, port, "127.0.0.1",
                                                   dpath, false, false, logdir, seed, opt);
  // Singular values: run() keeps them in a local; recompute them from the
  // final bidiagonal with the same bisection run() used (client.cpp:966-985).
  int k = (int)std::min(m, c->global_n);
  double* a = c->x_diagonal;
  double* b = c->x_upper_diagonal;
  int cnt = negative_count(k, a, b, pow(cblas_dnrm2(k, a, 1), 2) + pow(cblas_dnrm2(k - 1, b, 1), 2)) -
            negative_count(k, a, b, 0);
  if (topk > 0 && topk < cnt) cnt = topk;
  double* sig = new double[cnt > 0 ? cnt : 1]();
  if (mode == 0 || mode == 4) {   // dbdsdc left the singular values in x_diagonal
    for (int i = 0; i < cnt; ++i) sig[i] = a[i];
  } else {
    int got = 0;
    double bound = pow(cblas_dnrm2(k, a, 1), 2) + pow(cblas_dnrm2(k - 1, b, 1), 2);
    bisection_singular_values(k, a, b, 0, bound, 1e-20, cnt, sig, &got);
  }
  dump(out + "/sigma.bin", sig, cnt);
  // FinalU / FinalVT are left unset by the reference in the modes that skip
  // them (svd_mode 3 / 2, client.cpp:491-492)
  if (cid == 0 && mode != 3 && mode != 4) dump(out + "/U.bin", c->FinalU, m * (size_t)cnt);
  if (mode != 2 && mode != 4) dump(out + "/VT.bin", c->FinalVT, (size_t)cnt * ln);
  if (mode == 4) dump(out + "/w.bin", c->w_lr, ln);
  if (mode != 0 && mode != 4) {
    dump(out + "/ab.bin", a, k);
    FILE* fp = fopen((out + "/ab.bin").c_str(), "ab");
    fwrite(b, sizeof(double), k - 1, fp);
    fclose(fp);
  }
  FILE* ft = fopen((out + "/time.txt").c_str(), "w");
  fprintf(ft, "%.9f %.9f %.9f %.9f %.9f %.9f %.9f %.9f %.9f\n", time_diff(c->run_begin, c->run_finish),
          c->time_local_qr, c->time_global_qr, c->time_apply_mask, c->time_exchange_low_dim,
          c->time_bi_diag, c->time_bsvd, c->time_combine_svd_remove_mask, c->time_communication);
  fclose(ft);
  fflush(stdout);
  // Give peers time to drain their sockets before this process closes its
  // end; the reference's destructor joins a server thread that only ends
  // when every peer has disconnected.
  sleep(1);
  _exit(0);
}
