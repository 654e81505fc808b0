// ghb_log.hpp — per-call tracing of the public operator entry points.
//
// Every call opens an NVTX range named for the operator (free unless an
// Nsight tool is attached).  A context whose log is open (ghb_ctx_set_log,
// or GHB_LOG=<path> and GHB_LOG_LEVEL at ghb_ctx_create) also gets one JSON
// line per call in that file:
//   level 1: {"op", "device", "rows", "bytes", "host_us", "status"}: host_us is
//            the call's own time (the enqueue of an asynchronous call, the
//            whole call for the host-buffer and plan entry points);
//   level 2: an asynchronous call is also bracketed by CUDA events on its
//            stream and waits for them, adding "device_us", "gbs" (bytes /
//            device_us) and, when the log was given a peak, "roofline_frac";
//            a synchronous call reports its host time as "device_us".
// "bytes" are the call's algorithmic input bytes: every row of every input
// column it is given, at the column's width.  Level 2 synchronises each
// call, so it is for measurement, not for production or stream capture.
#pragma once

#include <nvtx3/nvToolsExt.h>

#include <chrono>

#include "ghb_ctx.hpp"

namespace ghb {

// Bytes of n rows of each column (a STRING column: its pairs).
inline int64_t cols_bytes(const ghb_column* cols, int32_t ncols) {
  int64_t b = 0;
  for (int i = 0; cols && i < ncols; i++) b += cols[i].n * (int64_t)type_width(cols[i].type);
  return b;
}

// One call's NVTX range and log line.  An asynchronous call (on `stream`)
// is timed by events at level 2; a synchronous one (host-buffer and plan
// entry points, `synchronous` set) by its own host time, which then covers
// its copies and kernels.
class CallScope {
 public:
  CallScope(ghb_ctx* ctx, const char* op, cudaStream_t stream, bool synchronous = false)
      : ctx_(ctx), op_(op), stream_(stream), sync_(synchronous) {
    nvtxRangePushA(op);
    if (!ctx_ || !ctx_->log) return;
    t0_ = std::chrono::steady_clock::now();
    if (!sync_ && ctx_->log_level >= 2 && ctx_->log_ev[0])
      timed_ = cudaEventRecord(ctx_->log_ev[0], stream_) == cudaSuccess;
  }
  ~CallScope() {
    if (ctx_ && ctx_->log) write();
    nvtxRangePop();
  }
  CallScope(const CallScope&) = delete;
  CallScope& operator=(const CallScope&) = delete;
  void rows(int64_t r) { rows_ = r; }
  void bytes(int64_t b) { bytes_ = b; }
  int32_t done(int32_t st) {
    status_ = st;
    return st;
  }

 private:
  void write() {
    double dev_us = -1;
    if (timed_ && status_ == GHB_OK && cudaEventRecord(ctx_->log_ev[1], stream_) == cudaSuccess &&
        cudaEventSynchronize(ctx_->log_ev[1]) == cudaSuccess) {
      float ms = 0;
      if (cudaEventElapsedTime(&ms, ctx_->log_ev[0], ctx_->log_ev[1]) == cudaSuccess) dev_us = ms * 1e3;
    }
    cudaGetLastError();
    const double host_us =
        std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0_).count();
    if (sync_ && ctx_->log_level >= 2 && status_ == GHB_OK) dev_us = host_us;
    std::fprintf(ctx_->log, "{\"op\": \"%s\", \"device\": %d, \"rows\": %lld, \"bytes\": %lld, \"host_us\": %.1f",
                 op_, ctx_->device, (long long)rows_, (long long)bytes_, host_us);
    if (dev_us > 0) {
      const double gbs = (double)bytes_ / (dev_us * 1e3);
      std::fprintf(ctx_->log, ", \"device_us\": %.1f, \"gbs\": %.6g", dev_us, gbs);
      if (ctx_->log_peak_gbs > 0) std::fprintf(ctx_->log, ", \"roofline_frac\": %.6g", gbs / ctx_->log_peak_gbs);
    }
    std::fprintf(ctx_->log, ", \"status\": %d}\n", status_);
  }

  ghb_ctx* ctx_;
  const char* op_;
  cudaStream_t stream_;
  bool sync_;
  std::chrono::steady_clock::time_point t0_{};
  bool timed_ = false;
  int64_t rows_ = 0, bytes_ = 0;
  int32_t status_ = GHB_OK;
};

}  // namespace ghb
