// ghb_jit.cu — group-by fold kernels compiled at run time for one signature.
//
// The generic fold (fold_tile) decides per row what the predicate nodes,
// the key column and each accumulator are; a launch's signature fixes all of
// that, and the generic kernel spends much of its instructions on those
// decisions (one warp instruction in four is a branch).  For a call's
// signature this file writes the type that names it (SigFolder<...> from
// ghb_gb_sig.cuh), compiles a kernel instantiating fold_kernel_body (or
// batch_fold_body) with it by NVRTC for sm_100a, loads the cubin with the
// runtime's library API and caches it by signature, in memory and on disk
// ($GHB_JIT_CACHE, default ~/.cache/ghive_b200/jit).  Literal values stay in
// the kernel parameters, so calls that differ only in literals share a kernel.
// GHB_JIT=0 in the environment turns this off (the generic kernels run).  A
// signature whose compilation fails falls back to the generic kernel.
#include <nvrtc.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdlib>
#include <fstream>
#include <iterator>
#include <mutex>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "ghb_groupby.cuh"

// Header sources embedded at build time (generated by ghive_b200/build.py).
extern const int ghb_jit_nheaders;
extern const char* const ghb_jit_header_names[];
extern const char* const ghb_jit_header_srcs[];

namespace ghb {

namespace {

// The fixed-width integer names the headers use; NVRTC has no libc headers.
const char* kStdintShim =
    "#pragma once\n"
    "typedef signed char int8_t; typedef short int16_t; typedef int int32_t; typedef long long int64_t;\n"
    "typedef unsigned char uint8_t; typedef unsigned short uint16_t; typedef unsigned int uint32_t;\n"
    "typedef unsigned long long uint64_t; typedef long long intptr_t; typedef unsigned long long uintptr_t;\n"
    "#define INT32_MAX 2147483647\n#define INT32_MIN (-INT32_MAX - 1)\n"
    "#define INT64_MAX 9223372036854775807LL\n#define INT64_MIN (-INT64_MAX - 1)\n"
    "#define UINT64_MAX 18446744073709551615ULL\n";

std::string col_t(const GbParams& p, int c) {
  std::ostringstream o;
  o << "ghb::ColT<" << c << ", " << p.cols.c[c].type << ", " << p.cols.c[c].null_mode << ">";
  return o.str();
}

// The predicate node k of the (post-order) program as a type.
std::string pred_t(const GbParams& p, int k) {
  const ghb_pred_node& nd = p.pred.nodes[k];
  std::ostringstream o;
  if (nd.mode == GHB_FILTER_AND || nd.mode == GHB_FILTER_OR) {
    o << (nd.mode == GHB_FILTER_AND ? "ghb::PAnd<" : "ghb::POr<") << pred_t(p, nd.child[0]) << ", "
      << pred_t(p, nd.child[1]) << ">";
  } else if (nd.col2 >= 0 && nd.mode != GHB_FILTER_NOT_NULL) {
    o << "ghb::PCols<" << nd.mode << ", " << col_t(p, nd.col) << ", " << col_t(p, nd.col2) << ">";
  } else {
    o << "ghb::PLeaf<" << k << ", " << nd.mode << ", " << col_t(p, nd.col) << ", "
      << (nd.lit_is_double ? "true" : "false") << ">";
  }
  return o.str();
}

uint64_t fnv1a(const std::string& s, uint64_t h = 1469598103934665603ull) {
  for (unsigned char c : s) {
    h ^= c;
    h *= 1099511628211ull;
  }
  return h;
}

struct Entry {
  cudaLibrary_t lib = nullptr;
  cudaKernel_t kern = nullptr;
  bool failed = false;
};

std::mutex g_mu;
std::unordered_map<std::string, Entry> g_cache;   // key: device + source

std::string cache_dir() {
  const char* d = std::getenv("GHB_JIT_CACHE");
  if (d && *d) return d;
  const char* home = std::getenv("HOME");
  return std::string(home && *home ? home : "/tmp") + "/.cache/ghive_b200/jit";
}

void mkdirs(const std::string& path) {
  std::string cur;
  std::stringstream ss(path);
  std::string part;
  if (!path.empty() && path[0] == '/') cur = "/";
  while (std::getline(ss, part, '/')) {
    if (part.empty()) continue;
    cur += part + "/";
    mkdir(cur.c_str(), 0755);
  }
}

}  // namespace

bool jit_enabled() {
  const char* e = std::getenv("GHB_JIT");
  return !(e && e[0] == '0');
}

// The kernel source for a signature: `batch` selects the batched fold,
// `threads` is the CTA size (with p.tile_rows it fixes the rows per thread).
std::string jit_groupby_source(const GbParams& p, bool keyed, bool batch, int threads) {
  std::ostringstream o;
  o << "#include \"ghb_gb_sig.cuh\"\n";
  o << "using Sig = ghb::SigFolder<" << p.tile_rows / std::max(1, threads) << ", "
    << (!keyed ? 0 : batch ? 2 : p.warp_agg ? 1 : 0) << ", " << (keyed ? "true" : "false") << ", "
    << (keyed ? col_t(p, p.key_col) : std::string("ghb::NoCol")) << ", "
    << (p.pred.n_nodes ? pred_t(p, p.pred.n_nodes - 1) : std::string("ghb::PTrue"));
  for (int a = 0; a < p.acc.n_acc; a++)
    o << ", ghb::AccT<" << (int)p.acc.kind[a] << ", "
      << (p.acc.col[a] >= 0 ? col_t(p, p.acc.col[a]) : std::string("ghb::NoCol")) << ">";
  o << ">;\n";
  // (1024, 1): shared memory holds these CTAs to one or two per SM anyway, so
  // the register budget is 64 per thread, not the 32 of two full CTAs
  if (batch)
    o << "extern \"C\" __global__ void __launch_bounds__(1024, 1) ghb_jit_fold(ghb::BatchParams bp) {\n"
         "  ghb::batch_fold_body<Sig>(bp);\n}\n";
  else
    o << "extern \"C\" __global__ void __launch_bounds__(1024, 1) ghb_jit_fold(ghb::GbParams p) {\n"
         "  ghb::fold_kernel_body<Sig>(p);\n}\n";
  return o.str();
}

// Compiles `src` to a sm_100a cubin; false (and the compiler log) on failure.
bool jit_compile(const std::string& src, std::vector<char>* cubin, std::string* log) {
  std::vector<const char*> names, srcs;
  for (int i = 0; i < ghb_jit_nheaders; i++) {
    names.push_back(ghb_jit_header_names[i]);
    srcs.push_back(ghb_jit_header_srcs[i]);
  }
  names.push_back("stdint.h");
  srcs.push_back(kStdintShim);
  nvrtcProgram prog;
  if (nvrtcCreateProgram(&prog, src.c_str(), "ghb_jit_fold.cu", (int)names.size(), srcs.data(), names.data()) !=
      NVRTC_SUCCESS) {
    if (log) *log = "nvrtcCreateProgram failed";
    return false;
  }
  // -default-device: the public header's C function declarations (host API,
  // never called here) are read as device declarations
  const char* opts[] = {"--gpu-architecture=sm_100a", "-std=c++17", "-lineinfo", "-default-device"};
  nvrtcResult r = nvrtcCompileProgram(prog, 4, opts);
  size_t ls = 0;
  nvrtcGetProgramLogSize(prog, &ls);
  if (log) {
    log->assign(ls, '\0');
    if (ls) nvrtcGetProgramLog(prog, &(*log)[0]);
  }
  bool ok = r == NVRTC_SUCCESS;
  if (ok) {
    size_t n = 0;
    ok = nvrtcGetCUBINSize(prog, &n) == NVRTC_SUCCESS && n > 0;
    if (ok) {
      cubin->resize(n);
      ok = nvrtcGetCUBIN(prog, cubin->data()) == NVRTC_SUCCESS;
    }
  }
  nvrtcDestroyProgram(&prog);
  return ok;
}

// The specialised fold kernel for a signature on the current device, or
// nullptr (then the caller runs the generic kernel).  Compiles on first use.
const void* jit_groupby_kernel(const GbParams& p, bool keyed, bool batch, int threads) {
  if (!jit_enabled()) return nullptr;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  if (threads <= 0 || p.tile_rows % threads || p.tile_rows / threads < 1 || p.tile_rows / threads > kGbRows)
    return nullptr;
  const std::string src = jit_groupby_source(p, keyed, batch, threads);
  const std::string key = std::to_string(dev) + "\n" + src;
  std::lock_guard<std::mutex> g(g_mu);
  auto it = g_cache.find(key);
  if (it != g_cache.end()) return it->second.failed ? nullptr : (const void*)it->second.kern;
  Entry e;
  // a cubin compiled earlier, by source, header and compiler version
  uint64_t h = fnv1a(src);
  for (int i = 0; i < ghb_jit_nheaders; i++) h = fnv1a(ghb_jit_header_srcs[i], h);
  int maj = 0, min = 0;
  nvrtcVersion(&maj, &min);
  h = fnv1a(std::to_string(maj) + "." + std::to_string(min), h);
  char name[64];
  snprintf(name, sizeof(name), "/fold_%016llx.cubin", (unsigned long long)h);
  const std::string path = cache_dir() + name;
  std::vector<char> cubin;
  {
    std::ifstream f(path, std::ios::binary);
    if (f) cubin.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  }
  if (cubin.empty()) {
    std::string log;
    if (jit_compile(src, &cubin, &log)) {
      mkdirs(cache_dir());
      const std::string tmp = path + ".tmp" + std::to_string((long long)getpid());
      std::ofstream f(tmp, std::ios::binary);
      f.write(cubin.data(), (std::streamsize)cubin.size());
      f.close();
      if (f) std::rename(tmp.c_str(), path.c_str());
    } else {
      cubin.clear();
    }
  }
  if (cubin.empty() ||
      cudaLibraryLoadData(&e.lib, cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0) != cudaSuccess ||
      cudaLibraryGetKernel(&e.kern, e.lib, "ghb_jit_fold") != cudaSuccess) {
    cudaGetLastError();
    e.failed = true;
  }
  g_cache[key] = e;
  return e.failed ? nullptr : (const void*)e.kern;
}

}  // namespace ghb

using namespace ghb;

extern "C" int32_t ghb_jit_groupby_source(const ghb_predicate* pred, const ghb_column* cols, int32_t ncols,
                                          const int32_t* key_cols, int32_t nkeys, const ghb_agg_desc* aggs,
                                          int32_t naggs, int32_t batch, char* buf, int64_t len) {
  if (!buf || len < 1) return GHB_ERR_INVALID;
  if (nkeys < 0 || nkeys > 1 || naggs < 0 || naggs > kMaxAggs || ncols < 0 || ncols > kMaxCols)
    return GHB_ERR_INVALID;
  // host-side planning only: a context object without device state, and
  // output descriptors with the result types and a placeholder address
  ghb_ctx local;
  ghb_out_column out[1 + kMaxAggs];
  std::memset(out, 0, sizeof(out));
  static char placeholder[8];
  for (int k = 0; k < nkeys; k++) {
    if (!key_cols || key_cols[k] < 0 || key_cols[k] >= ncols) return GHB_ERR_INVALID;
    out[k].type = cols[key_cols[k]].type;
    out[k].data = placeholder;
  }
  for (int a = 0; a < naggs; a++) {
    const int c = aggs[a].col;
    const int in = (c >= 0 && c < ncols) ? cols[c].type : GHB_LONG;
    int t = in;
    if (aggs[a].type == GHB_AGG_CNT) t = GHB_LONG;
    else if (aggs[a].type == GHB_AGG_AVG) t = GHB_DOUBLE;
    else if (aggs[a].type == GHB_AGG_SUM) t = in == GHB_DOUBLE ? GHB_DOUBLE : GHB_LONG;
    out[nkeys + a].type = t;
    out[nkeys + a].data = placeholder;
  }
  GbSetup su{};
  su.warp_agg = -1;
  GbParams p;
  FinParams f;
  size_t tb = 0, smem = 0;
  int64_t d_groups = 0;
  int32_t st = gb_setup(&local, pred, cols, ncols, key_cols, nkeys, aggs, naggs, out, 1 << 20, &d_groups, su, &p,
                        &f, &tb, &smem);
  if (st) return st;
  const std::string s = jit_groupby_source(p, nkeys == 1, batch != 0, kGbThreads);
  const size_t n = std::min<size_t>((size_t)len - 1, s.size());
  std::memcpy(buf, s.data(), n);
  buf[n] = 0;
  return s.size() < (size_t)len ? GHB_OK : GHB_ERR_CAPACITY;
}

extern "C" int32_t ghb_jit_compile_source(const char* source, int64_t* cubin_bytes, char* log, int64_t len) {
  if (!source) return GHB_ERR_INVALID;
  std::vector<char> cubin;
  std::string lg;
  const bool ok = jit_compile(source, &cubin, &lg);
  if (cubin_bytes) *cubin_bytes = (int64_t)cubin.size();
  if (log && len > 0) {
    const size_t n = std::min<size_t>((size_t)len - 1, lg.size());
    std::memcpy(log, lg.data(), n);
    log[n] = 0;
  }
  return ok ? GHB_OK : GHB_ERR_UNSUPPORTED;
}
