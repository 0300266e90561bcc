// Host-side entries of the whole pipeline (include/bbtsvd_b200.h):
//
//   bbt_fedsvd_run_host   host buffers in and out;
//   bbt_fedsvd_run_files  the reference's on-disk input, dpath/Client<c>.mat
//                         (and dpath/y.mat for svd_mode 4), as its participants
//                         load it (client.cpp:210-213, 1028; utils.cpp:237-252).
//
// Both stage the P blocks into a device arena kept by the context and overlap
// the copies with the pipeline: participant c's H2D runs on a copy stream and
// gates only the work on participant c (ctx->in_ready[c]); FinalVT_c leaves on
// a second copy stream as soon as it is computed (ctx->vt_done[c]).
//
// The file entry reads on a host thread through two pinned staging buffers,
// so file c+1 is read while the GPU works on participant c.  The pipeline
// waits on a host-side gate (ctx->io_gate) before it orders its stream after
// in_ready[c], so no stream ever waits on an event that is not recorded yet.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <cerrno>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

namespace bbt {

bbt_status wait_input(bbt_ctx* ctx, int c) {
  if (ctx->io_gate && !ctx->io_gate(ctx->io_gate_arg, c))
    return fail(ctx, BBT_ERR_IO, "fedsvd: the input of participant %d could not be read", c);
  BBT_CUDA(ctx, cudaStreamWaitEvent(ctx->stream, ctx->in_ready[c], 0));
  return BBT_OK;
}

namespace {

constexpr size_t STAGE_BYTES = (size_t)64 << 20;   // one pinned staging buffer (two are kept)

struct IoBufs {
  std::vector<double*> dX, dVT;
  double *ds = nullptr, *dU = nullptr, *dy = nullptr;
};

// Device staging of the inputs and outputs in the context's io arena (grows,
// never shrinks), the copy streams and the per-participant events.
bbt_status io_prepare(bbt_ctx* ctx, const bbt_fedsvd_config* cfg, bool want_v, bool lr, IoBufs& b) {
  const int P = cfg->participants;
  const size_t m = cfg->m;
  size_t gn = 0;
  for (int c = 0; c < P; ++c) gn += cfg->local_n[c];
  const size_t kmax = std::min(m, gn);   // singular values: the bidiagonal's order
  size_t need = (m + 2 * kmax + m * kmax) * sizeof(double) + 8192;
  for (int c = 0; c < P; ++c) need += (want_v ? 2 : 1) * (m * cfg->local_n[c] * sizeof(double) + 256);
  if (ctx->io_ws.cap < need) BBT_CUDA(ctx, ctx->io_ws.reserve(need));
  ctx->io_ws.reset();
  b.dX.assign(P, nullptr);
  b.dVT.assign(P, nullptr);
  for (int c = 0; c < P; ++c) {
    b.dX[c] = ctx->io_ws.take<double>(m * cfg->local_n[c]);
    if (want_v) b.dVT[c] = ctx->io_ws.take<double>(m * cfg->local_n[c]);
  }
  b.ds = ctx->io_ws.take<double>(kmax);
  b.dU = ctx->io_ws.take<double>(m * kmax);
  if (lr) b.dy = ctx->io_ws.take<double>(m);
  if (!b.dU || (lr && !b.dy)) return fail(ctx, BBT_ERR_NOMEM, "fedsvd: host-entry staging");
  if (!ctx->copy_in) BBT_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->copy_in, cudaStreamNonBlocking));
  if (!ctx->copy_out) BBT_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->copy_out, cudaStreamNonBlocking));
  while ((int)ctx->in_ready.size() < P) {
    cudaEvent_t a, e;
    BBT_CUDA(ctx, cudaEventCreateWithFlags(&a, cudaEventDisableTiming));
    BBT_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    ctx->in_ready.push_back(a);
    ctx->vt_done.push_back(e);
  }
  // the copy streams start after all earlier work on the context's stream
  BBT_CUDA(ctx, cudaEventRecord(ctx->vt_done[0], ctx->stream));
  BBT_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_in, ctx->vt_done[0], 0));
  BBT_CUDA(ctx, cudaStreamWaitEvent(ctx->copy_out, ctx->vt_done[0], 0));
  return BBT_OK;
}

// Run the pipeline on the staged inputs; sigma and FinalU are copied out at
// the end, every FinalVT_c (or w_c) by the pipeline as soon as it is done.
bbt_status io_run(bbt_ctx* ctx, const bbt_fedsvd_config* dcfg, IoBufs& b, double* hsigma, double* hU,
                  double* const* hVT, int* k, bool want_u, bool want_v) {
  const int P = dcfg->participants;
  ctx->vt_dst.assign(P, nullptr);
  if (want_v)
    for (int c = 0; c < P; ++c) ctx->vt_dst[c] = hVT[c];
  ctx->io_on = true;
  bbt_status st = fedsvd(ctx, dcfg, b.dX.data(), b.ds, b.dU, b.dVT.data(), k);
  ctx->io_on = false;
  if (st != BBT_OK) return st;
  const int kk = *k;
  cudaError_t e = cudaMemcpyAsync(hsigma, b.ds, kk * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess && want_u)
    e = cudaMemcpyAsync(hU, b.dU, dcfg->m * kk * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "fedsvd: copy-out");
  return BBT_OK;
}

// Every copy issued on the copy streams has finished before the buffers may be reused.
bbt_status io_drain(bbt_ctx* ctx, bbt_status st) {
  const cudaError_t e1 = cudaStreamSynchronize(ctx->copy_in), e2 = cudaStreamSynchronize(ctx->copy_out);
  if (st == BBT_OK && e1 != cudaSuccess) st = cuda_fail(ctx, e1, "fedsvd: copy-in");
  if (st == BBT_OK && e2 != cudaSuccess) st = cuda_fail(ctx, e2, "fedsvd: copy-out");
  return st;
}

bbt_status check_host_args(bbt_ctx* ctx, const bbt_fedsvd_config* cfg, double* hsigma, double* hU,
                           double* const* hVT, int* k, bool& want_u, bool& want_v, bool& lr) {
  if (!cfg || !k || !hsigma || cfg->participants < 1 || !cfg->local_n || !cfg->private_seeds)
    return fail(ctx, BBT_ERR_ARG, "fedsvd: NULL argument");
  lr = cfg->svd_mode == 4;
  want_u = cfg->svd_mode != 3 && !lr;
  want_v = cfg->svd_mode != 2;
  if ((want_u && !hU) || (want_v && !hVT)) return fail(ctx, BBT_ERR_ARG, "fedsvd: NULL output");
  if (want_v)
    for (int c = 0; c < cfg->participants; ++c)
      if (!hVT[c]) return fail(ctx, BBT_ERR_ARG, "fedsvd: NULL output of participant %d", c);
  return BBT_OK;
}

// ---- the on-disk input --------------------------------------------------

struct Reader {
  std::mutex mu;
  std::condition_variable cv;
  int done = 0;            // participants whose input has been read and its copy enqueued
  bool failed = false;
  std::string msg;
  std::atomic<bool> cancel{false};
};

bool gate(void* arg, int c) {
  Reader* r = static_cast<Reader*>(arg);
  std::unique_lock<std::mutex> lk(r->mu);
  r->cv.wait(lk, [&] { return r->done > c || r->failed; });
  return r->done > c;
}

// pread of len bytes at off into dst, split over up to `threads` threads.
bool pread_all(int fd, char* dst, size_t len, off_t off, int threads, std::string& msg) {
  std::vector<std::thread> th;
  std::atomic<bool> ok{true};
  std::atomic<int> err{0};
  const size_t piece = std::max<size_t>((len / threads + 4095) & ~size_t(4095), (size_t)4 << 20);
  auto work = [&](size_t a, size_t b) {
    while (a < b && ok) {
      const ssize_t r = pread(fd, dst + a, b - a, off + (off_t)a);
      if (r <= 0) {
        ok = false;
        err = r < 0 ? errno : 0;
        return;
      }
      a += (size_t)r;
    }
  };
  for (size_t a = piece; a < len; a += piece) th.emplace_back(work, a, std::min(len, a + piece));
  work(0, std::min(len, piece));
  for (auto& t : th) t.join();
  if (!ok) msg = err ? std::strerror(err) : "unexpected end of file";
  return ok;
}

struct FileJob {
  std::string path;
  size_t bytes;
  double* dst;
};

// Reader thread: file after file, chunk after chunk through the two pinned
// staging buffers; in_ready[c] is recorded after participant c's file (and
// after y.mat for the last participant), then the gate opens for c.
void read_inputs(bbt_ctx* ctx, std::vector<std::vector<FileJob>> jobs, Reader* R) {
  cudaSetDevice(ctx->device);
  const int threads = (int)std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
  size_t chunk = 0;
  auto failed = [&](const std::string& m) {
    std::lock_guard<std::mutex> lk(R->mu);
    R->failed = true;
    R->msg = m;
    R->cv.notify_all();
  };
  for (size_t c = 0; c < jobs.size(); ++c) {
    for (const FileJob& j : jobs[c]) {
      const int fd = open(j.path.c_str(), O_RDONLY);
      if (fd < 0) return failed(j.path + ": " + std::strerror(errno));
      for (size_t off = 0; off < j.bytes; off += STAGE_BYTES, ++chunk) {
        if (R->cancel) {
          close(fd);
          return failed("cancelled");
        }
        const int s = (int)(chunk & 1);
        const size_t len = std::min(STAGE_BYTES, j.bytes - off);
        char* stage = static_cast<char*>(ctx->io_pinned) + s * STAGE_BYTES;
        cudaError_t e = cudaEventSynchronize(ctx->io_stage_ev[s]);   // its previous copy has left
        std::string msg;
        if (e == cudaSuccess && !pread_all(fd, stage, len, (off_t)off, threads, msg)) {
          close(fd);
          return failed(j.path + ": " + msg);
        }
        if (e == cudaSuccess)
          e = cudaMemcpyAsync(reinterpret_cast<char*>(j.dst) + off, stage, len, cudaMemcpyHostToDevice,
                              ctx->copy_in);
        if (e == cudaSuccess) e = cudaEventRecord(ctx->io_stage_ev[s], ctx->copy_in);
        if (e != cudaSuccess) {
          close(fd);
          return failed(std::string("H2D copy: ") + cudaGetErrorString(e));
        }
      }
      close(fd);
    }
    const cudaError_t e = cudaEventRecord(ctx->in_ready[c], ctx->copy_in);
    if (e != cudaSuccess) return failed(std::string("event: ") + cudaGetErrorString(e));
    std::lock_guard<std::mutex> lk(R->mu);
    R->done = (int)c + 1;
    R->cv.notify_all();
  }
}

}  // namespace
}  // namespace bbt

using namespace bbt;

extern "C" {

bbt_status bbt_fedsvd_run_host(bbt_ctx* ctx, const bbt_fedsvd_config* cfg, const double* const* hX,
                               double* hsigma, double* hU, double* const* hVT, int* k) {
  if (!ctx) return BBT_ERR_ARG;
  bool want_u, want_v, lr;
  BBT_TRY(check_host_args(ctx, cfg, hsigma, hU, hVT, k, want_u, want_v, lr));
  if (!hX || (lr && !cfg->labels)) return fail(ctx, BBT_ERR_ARG, "fedsvd_host: NULL input");
  const int P = cfg->participants;
  const size_t m = cfg->m;
  IoBufs b;
  BBT_TRY(io_prepare(ctx, cfg, want_v, lr, b));
  for (int c = 0; c < P; ++c) {   // participant by participant: the first QR starts after one block
    BBT_CUDA(ctx, cudaMemcpyAsync(b.dX[c], hX[c], m * cfg->local_n[c] * sizeof(double), cudaMemcpyHostToDevice,
                                  ctx->copy_in));
    if (lr && c == P - 1)   // the labels travel with the last participant's block
      BBT_CUDA(ctx, cudaMemcpyAsync(b.dy, cfg->labels, m * sizeof(double), cudaMemcpyHostToDevice, ctx->copy_in));
    BBT_CUDA(ctx, cudaEventRecord(ctx->in_ready[c], ctx->copy_in));
  }
  bbt_fedsvd_config dcfg = *cfg;
  dcfg.labels = b.dy;
  return io_drain(ctx, io_run(ctx, &dcfg, b, hsigma, hU, hVT, k, want_u, want_v));
}

bbt_status bbt_fedsvd_run_files(bbt_ctx* ctx, const bbt_fedsvd_config* cfg, const char* dpath, double* hsigma,
                                double* hU, double* const* hVT, int* k) {
  if (!ctx) return BBT_ERR_ARG;
  bool want_u, want_v, lr;
  BBT_TRY(check_host_args(ctx, cfg, hsigma, hU, hVT, k, want_u, want_v, lr));
  if (!dpath) return fail(ctx, BBT_ERR_ARG, "fedsvd_files: NULL path");
  const int P = cfg->participants;
  const size_t m = cfg->m;
  // every file is checked before any work starts (client.cpp:211, 1028)
  std::vector<std::vector<FileJob>> jobs(P);
  for (int c = 0; c < P; ++c) {
    const std::string f = std::string(dpath) + "/Client" + std::to_string(c) + ".mat";
    jobs[c].push_back({f, m * cfg->local_n[c] * sizeof(double), nullptr});
  }
  if (lr) jobs[P - 1].push_back({std::string(dpath) + "/y.mat", m * sizeof(double), nullptr});
  for (auto& js : jobs)
    for (auto& j : js) {
      struct stat sb;
      if (stat(j.path.c_str(), &sb) != 0)
        return fail(ctx, BBT_ERR_IO, "fedsvd_files: %s: %s", j.path.c_str(), std::strerror(errno));
      if ((size_t)sb.st_size != j.bytes)
        return fail(ctx, BBT_ERR_IO, "fedsvd_files: %s holds %lld bytes, expected %zu (float64)", j.path.c_str(),
                    (long long)sb.st_size, j.bytes);
    }
  IoBufs b;
  BBT_TRY(io_prepare(ctx, cfg, want_v, lr, b));
  for (int c = 0; c < P; ++c) jobs[c][0].dst = b.dX[c];
  if (lr) jobs[P - 1][1].dst = b.dy;
  if (!ctx->io_pinned) {
    BBT_CUDA(ctx, cudaHostAlloc(&ctx->io_pinned, 2 * STAGE_BYTES, cudaHostAllocDefault));
    for (auto& e : ctx->io_stage_ev) BBT_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  Reader R;
  ctx->io_gate = gate;
  ctx->io_gate_arg = &R;
  std::thread reader(read_inputs, ctx, jobs, &R);
  bbt_fedsvd_config dcfg = *cfg;
  dcfg.labels = b.dy;
  bbt_status st = io_run(ctx, &dcfg, b, hsigma, hU, hVT, k, want_u, want_v);
  R.cancel = true;   // only matters when the pipeline stopped early
  reader.join();
  ctx->io_gate = nullptr;
  ctx->io_gate_arg = nullptr;
  if (R.failed && R.msg != "cancelled") {
    io_drain(ctx, BBT_OK);
    return fail(ctx, BBT_ERR_IO, "fedsvd_files: %s", R.msg.c_str());
  }
  return io_drain(ctx, st);
}

}  // extern "C"
