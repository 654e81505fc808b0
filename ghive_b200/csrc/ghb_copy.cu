// ghb_copy.cu — copies between pageable host memory and the device.
//
// GHive's JNI inputs are JVM direct buffers: pageable memory, which the CUDA
// driver copies at about 10 GB/s on this machine, while pinned memory moves
// at the link's 55 GB/s.  A copy of pageable memory goes instead through
// pinned staging buffers in lanes: each lane (a host thread) takes a
// contiguous share of the bytes and moves it in pieces through its own two
// buffers, so the host copy of one piece overlaps the DMA of the previous
// one and the lanes' host copies run side by side.  Pinned (or registered)
// memory and small copies go by one cudaMemcpyAsync.
#include <algorithm>
#include <thread>

#include "ghb_ctx.hpp"

namespace ghb {

bool host_pinned(const void* p) {
  cudaPointerAttributes attr;
  const bool pinned = cudaPointerGetAttributes(&attr, p) == cudaSuccess && attr.type == cudaMemoryTypeHost;
  cudaGetLastError();
  return pinned;
}

namespace {

constexpr size_t kSmallCopy = 1u << 20;   // below this the driver's own staging

int32_t ensure_staging(ghb_ctx* ctx) {
  for (int l = 0; l < kStageLanes; l++)
    for (int b = 0; b < 2; b++) {
      if (!ctx->stage[l][b] && cudaMallocHost(&ctx->stage[l][b], kStagePiece) != cudaSuccess) {
        cudaGetLastError();
        ctx->stage[l][b] = nullptr;
        return set_error(ctx, GHB_ERR_OOM, "cannot allocate pinned staging memory");
      }
      if (!ctx->stage_ev[l][b])
        GHB_CUDA_TRY(ctx, cudaEventCreateWithFlags(&ctx->stage_ev[l][b], cudaEventDisableTiming));
    }
  return GHB_OK;
}

int lanes_for(size_t total) {
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t by_size = (total + kStagePiece - 1) / kStagePiece;
  return (int)std::max<size_t>(1, std::min<size_t>({(size_t)kStageLanes, (size_t)std::max(1u, hw / 2), by_size}));
}

// Calls fn(task, offset, length) for the pieces of lane `lane`'s share of the
// tasks' bytes laid end to end, in order, each piece within one task and at
// most kStagePiece long.
template <class Fn>
cudaError_t for_lane_pieces(const std::vector<CopyTask>& tasks, size_t total, int lane, int lanes, Fn fn) {
  const size_t lo = total * lane / lanes, hi = total * (lane + 1) / lanes;
  size_t base = 0;
  for (const CopyTask& t : tasks) {
    const size_t a = std::max(lo, base), e = std::min(hi, base + t.bytes);
    for (size_t off = a; off < e; off += kStagePiece) {
      const cudaError_t err = fn(t, off - base, std::min(kStagePiece, e - off));
      if (err != cudaSuccess) return err;
    }
    base += t.bytes;
  }
  return cudaSuccess;
}

// Runs lane(i) for i in [0, lanes): lane 0 on this thread, the others on
// their own threads (on the context's device); the first error wins.
template <class Lane>
cudaError_t run_lanes(ghb_ctx* ctx, int lanes, Lane lane) {
  std::vector<cudaError_t> err(lanes, cudaSuccess);
  std::vector<std::thread> th;
  for (int i = 1; i < lanes; i++)
    th.emplace_back([&, i] {
      err[i] = cudaSetDevice(ctx->device);
      if (err[i] == cudaSuccess) err[i] = lane(i);
    });
  err[0] = lane(0);
  for (std::thread& t : th) t.join();
  for (cudaError_t e : err)
    if (e != cudaSuccess) return e;
  return cudaSuccess;
}

}  // namespace

int32_t copy_h2d_many(ghb_ctx* ctx, const std::vector<CopyTask>& tasks, cudaStream_t stream) {
  std::vector<CopyTask> staged;
  size_t total = 0;
  for (const CopyTask& t : tasks) {
    if (t.bytes == 0) continue;
    if (t.bytes < kSmallCopy || host_pinned(t.src)) {
      GHB_CUDA_TRY(ctx, cudaMemcpyAsync(t.dst, t.src, t.bytes, cudaMemcpyHostToDevice, stream));
    } else {
      staged.push_back(t);
      total += t.bytes;
    }
  }
  if (staged.empty()) return GHB_OK;
  int32_t st = ensure_staging(ctx);
  if (st) return st;
  const int lanes = lanes_for(total);
  const cudaError_t e = run_lanes(ctx, lanes, [&](int l) {
    int b = 0;
    return for_lane_pieces(staged, total, l, lanes, [&](const CopyTask& t, size_t off, size_t len) {
      cudaError_t r = cudaEventSynchronize(ctx->stage_ev[l][b]);   // the buffer's last DMA is done
      if (r != cudaSuccess) return r;
      std::memcpy(ctx->stage[l][b], (const char*)t.src + off, len);
      r = cudaMemcpyAsync((char*)t.dst + off, ctx->stage[l][b], len, cudaMemcpyHostToDevice, stream);
      if (r == cudaSuccess) r = cudaEventRecord(ctx->stage_ev[l][b], stream);
      b ^= 1;
      return r;
    });
  });
  if (e != cudaSuccess) return set_error(ctx, GHB_ERR_CUDA, "host-to-device copy: %s", cudaGetErrorString(e));
  return GHB_OK;
}

int32_t copy_h2d(ghb_ctx* ctx, void* dst, const void* src, size_t bytes, cudaStream_t stream) {
  return copy_h2d_many(ctx, {CopyTask{dst, src, bytes}}, stream);
}

int32_t copy_d2h_many(ghb_ctx* ctx, const std::vector<CopyTask>& tasks, cudaStream_t stream) {
  std::vector<CopyTask> staged;
  size_t total = 0;
  for (const CopyTask& t : tasks) {
    if (t.bytes == 0) continue;
    if (t.bytes < kSmallCopy || host_pinned(t.dst)) {
      GHB_CUDA_TRY(ctx, cudaMemcpyAsync(t.dst, t.src, t.bytes, cudaMemcpyDeviceToHost, stream));
    } else {
      staged.push_back(t);
      total += t.bytes;
    }
  }
  if (!staged.empty()) {
    int32_t st = ensure_staging(ctx);
    if (st) return st;
    const int lanes = lanes_for(total);
    const cudaError_t e = run_lanes(ctx, lanes, [&](int l) {
      // a piece's DMA into one buffer runs while the previous piece is
      // copied out of the other
      int b = 0;
      char* pend_dst = nullptr;
      size_t pend_len = 0;
      int pend_b = 0;
      cudaError_t r = for_lane_pieces(staged, total, l, lanes, [&](const CopyTask& t, size_t off, size_t len) {
        cudaError_t q = cudaEventSynchronize(ctx->stage_ev[l][b]);   // the buffer is free
        if (q == cudaSuccess)
          q = cudaMemcpyAsync(ctx->stage[l][b], (const char*)t.src + off, len, cudaMemcpyDeviceToHost, stream);
        if (q == cudaSuccess) q = cudaEventRecord(ctx->stage_ev[l][b], stream);
        if (q == cudaSuccess && pend_dst) {
          q = cudaEventSynchronize(ctx->stage_ev[l][pend_b]);
          if (q == cudaSuccess) std::memcpy(pend_dst, ctx->stage[l][pend_b], pend_len);
        }
        pend_dst = (char*)t.dst + off;
        pend_len = len;
        pend_b = b;
        b ^= 1;
        return q;
      });
      if (r == cudaSuccess && pend_dst) {
        r = cudaEventSynchronize(ctx->stage_ev[l][pend_b]);
        if (r == cudaSuccess) std::memcpy(pend_dst, ctx->stage[l][pend_b], pend_len);
      }
      return r;
    });
    if (e != cudaSuccess) return set_error(ctx, GHB_ERR_CUDA, "device-to-host copy: %s", cudaGetErrorString(e));
  }
  GHB_CUDA_TRY(ctx, cudaStreamSynchronize(stream));
  return GHB_OK;
}

}  // namespace ghb
