// lcmx.cu -- C ABI of the B200 backward-induction solver.
//
// Owns: the CUDA context binding, NVRTC compilation of generated model code
// for sm_100a (in-process and on-disk cubin caches), kernel lookup and
// launches of the generated kernels, and the model-independent kernels that
// are compiled into this library by nvcc (non-finite counting; the FUES scan
// lives in fues.cu).  See include/lcmx.h for the contract.

#include <cuda.h>
#include <cuda_runtime.h>
#include <nvrtc.h>

#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "../../include/lcmx.h"

struct lcmx_module;

// Driver API entry points, resolved through the runtime
// (cudaGetDriverEntryPoint) so that the library loads on machines without a
// driver (build / CPU test hosts) and fails only when a context is created.
struct DriverApi {
  CUresult (*GetErrorString)(CUresult, const char**) = nullptr;
  CUresult (*ModuleLoadData)(CUmodule*, const void*) = nullptr;
  CUresult (*ModuleUnload)(CUmodule) = nullptr;
  CUresult (*ModuleGetFunction)(CUfunction*, CUmodule, const char*) = nullptr;
  CUresult (*FuncSetAttribute)(CUfunction, CUfunction_attribute, int) = nullptr;
  CUresult (*OccupancyMaxActiveBlocksPerMultiprocessor)(int*, CUfunction, int, size_t) = nullptr;
  CUresult (*LaunchKernel)(CUfunction, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned, unsigned,
                           CUstream, void**, void**) = nullptr;
  CUresult (*ModuleGetGlobal)(CUdeviceptr*, size_t*, CUmodule, const char*) = nullptr;
  CUresult (*FuncGetAttribute)(int*, CUfunction_attribute, CUfunction) = nullptr;
  bool ok = false;
};
static DriverApi g_drv;
static std::mutex g_drv_mu;

template <typename F>
static bool drv_get(const char* name, F& fn) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess || !p)
    return false;
  fn = reinterpret_cast<F>(p);
  return true;
}

static bool drv_init() {
  std::lock_guard<std::mutex> g(g_drv_mu);
  if (g_drv.ok) return true;
  bool ok = drv_get("cuGetErrorString", g_drv.GetErrorString) && drv_get("cuModuleLoadData", g_drv.ModuleLoadData) &&
            drv_get("cuModuleUnload", g_drv.ModuleUnload) && drv_get("cuModuleGetFunction", g_drv.ModuleGetFunction) &&
            drv_get("cuFuncSetAttribute", g_drv.FuncSetAttribute) &&
            drv_get("cuOccupancyMaxActiveBlocksPerMultiprocessor", g_drv.OccupancyMaxActiveBlocksPerMultiprocessor) &&
            drv_get("cuLaunchKernel", g_drv.LaunchKernel) && drv_get("cuModuleGetGlobal", g_drv.ModuleGetGlobal) &&
            drv_get("cuFuncGetAttribute", g_drv.FuncGetAttribute);
  g_drv.ok = ok;
  return ok;
}

struct lcmx_ctx {
  int device = 0;
  int sm_count = 0;
  std::string err;
  std::mutex mu;
  std::unordered_map<std::string, lcmx_module*> modules;
};

struct lcmx_module {
  lcmx_ctx* ctx = nullptr;
  CUmodule mod = nullptr;
  std::string key;
  std::mutex mu;
  std::unordered_map<std::string, CUfunction> funcs;
  // resident CTAs per SM of (kernel, block, dynamic shared bytes), with the
  // shared-memory attributes already set: two driver queries per launch saved
  std::map<std::tuple<CUfunction, int, int>, int> geometry;
  int refs = 1;
};

static thread_local std::string g_tls_err;

static int set_err(lcmx_ctx* ctx, int code, const std::string& msg) {
  if (ctx) {
    ctx->err = msg;
  }
  g_tls_err = msg;
  return code;
}

static std::string cu_msg(CUresult r) {
  const char* s = nullptr;
  if (g_drv.GetErrorString) g_drv.GetErrorString(r, &s);
  return s ? s : ("driver error " + std::to_string((int)r));
}

extern "C" const char* lcmx_last_error(const lcmx_ctx* ctx) {
  if (ctx) return ctx->err.c_str();
  return g_tls_err.c_str();
}

extern "C" int lcmx_ctx_create(int device, lcmx_ctx** out) {
  if (!out) return set_err(nullptr, LCMX_ERR_ARGS, "lcmx_ctx_create: out is NULL");
  *out = nullptr;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return set_err(nullptr, LCMX_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  e = cudaFree(nullptr);  // establish the primary context
  if (e != cudaSuccess) return set_err(nullptr, LCMX_ERR_CUDA, std::string("cudaFree(0): ") + cudaGetErrorString(e));
  if (!drv_init()) return set_err(nullptr, LCMX_ERR_CUDA, "could not resolve CUDA driver entry points");
  auto* ctx = new lcmx_ctx();
  ctx->device = device;
  cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
  *out = ctx;
  return LCMX_OK;
}

extern "C" int lcmx_ctx_destroy(lcmx_ctx* ctx) {
  if (!ctx) return LCMX_ERR_ARGS;
  {
    std::lock_guard<std::mutex> g(ctx->mu);
    for (auto& kv : ctx->modules) {
      if (kv.second->mod) g_drv.ModuleUnload(kv.second->mod);
      delete kv.second;
    }
    ctx->modules.clear();
  }
  delete ctx;
  return LCMX_OK;
}

extern "C" int lcmx_device_info(lcmx_ctx* ctx, int* sm_count, size_t* free_bytes, size_t* total_bytes) {
  if (!ctx) return set_err(nullptr, LCMX_ERR_ARGS, "lcmx_device_info: ctx is NULL");
  cudaSetDevice(ctx->device);
  if (sm_count) *sm_count = ctx->sm_count;
  size_t f = 0, t = 0;
  cudaError_t e = cudaMemGetInfo(&f, &t);
  if (e != cudaSuccess) return set_err(ctx, LCMX_ERR_CUDA, std::string("cudaMemGetInfo: ") + cudaGetErrorString(e));
  if (free_bytes) *free_bytes = f;
  if (total_bytes) *total_bytes = t;
  return LCMX_OK;
}

// ---------------------------------------------------------------- caching
static std::string cache_dir() {
  const char* d = getenv("LCMX_CACHE_DIR");
  std::string dir;
  if (d && *d) {
    dir = d;
  } else {
    const char* home = getenv("HOME");
    dir = std::string(home ? home : "/tmp") + "/.cache/pylcm_b200";
  }
  return dir;
}

static void mkdirs(const std::string& path) {
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

static bool read_file(const std::string& p, std::vector<char>& out) {
  std::ifstream f(p, std::ios::binary);
  if (!f) return false;
  out.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  return !out.empty();
}

static void write_file_atomic(const std::string& p, const std::vector<char>& data) {
  std::string tmp = p + ".tmp." + std::to_string(getpid());
  {
    std::ofstream f(tmp, std::ios::binary);
    if (!f) return;
    f.write(data.data(), (std::streamsize)data.size());
  }
  rename(tmp.c_str(), p.c_str());
}

static bool safe_key(const std::string& k) {
  if (k.empty() || k.size() > 200) return false;
  for (char c : k) {
    if (!(isalnum((unsigned char)c) || c == '_' || c == '-' || c == '.')) return false;
  }
  return true;
}

extern "C" int lcmx_module_compile(lcmx_ctx* ctx, const char* cuda_src, const char* key,
                                   const char* options, lcmx_module** out) {
  if (!ctx || !cuda_src || !key || !out) return set_err(ctx, LCMX_ERR_ARGS, "lcmx_module_compile: NULL argument");
  if (!safe_key(key)) return set_err(ctx, LCMX_ERR_ARGS, "lcmx_module_compile: key must be [A-Za-z0-9_.-]{1,200}");
  *out = nullptr;
  {
    std::lock_guard<std::mutex> g(ctx->mu);
    auto it = ctx->modules.find(key);
    if (it != ctx->modules.end()) {
      it->second->refs++;
      *out = it->second;
      return LCMX_OK;
    }
  }
  cudaSetDevice(ctx->device);
  std::vector<char> cubin;
  const std::string dir = cache_dir();
  const std::string path = dir + "/" + key + ".cubin";
  const bool use_disk = getenv("LCMX_NO_DISK_CACHE") == nullptr;
  if (!(use_disk && read_file(path, cubin))) {
    nvrtcProgram prog;
    nvrtcResult nr = nvrtcCreateProgram(&prog, cuda_src, (std::string(key) + ".cu").c_str(), 0, nullptr, nullptr);
    if (nr != NVRTC_SUCCESS) return set_err(ctx, LCMX_ERR_COMPILE, std::string("nvrtcCreateProgram: ") + nvrtcGetErrorString(nr));
    std::vector<std::string> opts = {"--gpu-architecture=sm_100a", "--std=c++17", "-lineinfo",
                                     "--device-as-default-execution-space"};
    if (options) {
      std::stringstream ss(options);
      std::string line;
      while (std::getline(ss, line, '\n')) {
        if (!line.empty()) opts.push_back(line);
      }
    }
    std::vector<const char*> copts;
    for (auto& o : opts) copts.push_back(o.c_str());
    nr = nvrtcCompileProgram(prog, (int)copts.size(), copts.data());
    if (nr != NVRTC_SUCCESS) {
      size_t n = 0;
      nvrtcGetProgramLogSize(prog, &n);
      std::string log(n, '\0');
      if (n) nvrtcGetProgramLog(prog, &log[0]);
      nvrtcDestroyProgram(&prog);
      return set_err(ctx, LCMX_ERR_COMPILE, "NVRTC compile failed for " + std::string(key) + ":\n" + log);
    }
    size_t n = 0;
    nr = nvrtcGetCUBINSize(prog, &n);
    if (nr != NVRTC_SUCCESS || n == 0) {
      nvrtcDestroyProgram(&prog);
      return set_err(ctx, LCMX_ERR_COMPILE, "nvrtcGetCUBINSize failed");
    }
    cubin.resize(n);
    nvrtcGetCUBIN(prog, cubin.data());
    nvrtcDestroyProgram(&prog);
    if (use_disk) {
      mkdirs(dir);
      write_file_atomic(path, cubin);
    }
  }
  CUmodule m = nullptr;
  CUresult r = g_drv.ModuleLoadData(&m, cubin.data());
  if (r != CUDA_SUCCESS) return set_err(ctx, LCMX_ERR_MODULE, "cuModuleLoadData: " + cu_msg(r));
  auto* mod = new lcmx_module();
  mod->ctx = ctx;
  mod->mod = m;
  mod->key = key;
  {
    std::lock_guard<std::mutex> g(ctx->mu);
    auto it = ctx->modules.find(key);
    if (it != ctx->modules.end()) {  // raced with another thread
      g_drv.ModuleUnload(m);
      delete mod;
      it->second->refs++;
      *out = it->second;
      return LCMX_OK;
    }
    ctx->modules[key] = mod;
  }
  *out = mod;
  return LCMX_OK;
}

extern "C" int lcmx_module_destroy(lcmx_module* mod) {
  if (!mod) return LCMX_ERR_ARGS;
  lcmx_ctx* ctx = mod->ctx;
  std::lock_guard<std::mutex> g(ctx->mu);
  if (--mod->refs > 0) return LCMX_OK;
  ctx->modules.erase(mod->key);
  if (mod->mod) g_drv.ModuleUnload(mod->mod);
  delete mod;
  return LCMX_OK;
}

static int get_func(lcmx_module* mod, const char* name, CUfunction* f) {
  std::lock_guard<std::mutex> g(mod->mu);
  auto it = mod->funcs.find(name);
  if (it != mod->funcs.end()) {
    *f = it->second;
    return LCMX_OK;
  }
  CUresult r = g_drv.ModuleGetFunction(f, mod->mod, name);
  if (r != CUDA_SUCCESS)
    return set_err(mod->ctx, LCMX_ERR_MODULE, std::string("kernel ") + name + " not found: " + cu_msg(r));
  mod->funcs[name] = *f;
  return LCMX_OK;
}

// A launch whose static plus dynamic shared memory exceeds the 48 KB default
// needs the dynamic part opted in first (the static part counts against it).
static CUresult opt_in_smem(CUfunction f, int dyn_bytes) {
  int stat = 0;
  if (g_drv.FuncGetAttribute(&stat, CU_FUNC_ATTRIBUTE_SHARED_SIZE_BYTES, f) != CUDA_SUCCESS) stat = 0;
  if ((long long)dyn_bytes + stat <= 48 * 1024) return CUDA_SUCCESS;
  const CUresult r = g_drv.FuncSetAttribute(f, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, dyn_bytes);
  if (r != CUDA_SUCCESS) return r;
  // such a kernel is limited by shared memory: ask for the largest carveout
  // so that as many CTAs fit per SM as its registers allow
  return g_drv.FuncSetAttribute(f, CU_FUNC_ATTRIBUTE_PREFERRED_SHARED_MEMORY_CARVEOUT, 100);
}

extern "C" int lcmx_occupancy(lcmx_module* mod, const char* kernel, int block, int smem_bytes, int* blocks_per_sm) {
  if (!mod || !kernel || !blocks_per_sm || block <= 0) return set_err(mod ? mod->ctx : nullptr, LCMX_ERR_ARGS, "lcmx_occupancy: bad args");
  CUfunction f;
  int rc = get_func(mod, kernel, &f);
  if (rc) return rc;
  opt_in_smem(f, smem_bytes);
  int n = 0;
  CUresult r = g_drv.OccupancyMaxActiveBlocksPerMultiprocessor(&n, f, block, (size_t)smem_bytes);
  if (r != CUDA_SUCCESS) return set_err(mod->ctx, LCMX_ERR_CUDA, "occupancy: " + cu_msg(r));
  *blocks_per_sm = n;
  return LCMX_OK;
}

static int launch_items(lcmx_module* mod, const char* kernel, const lcmx_launch_args* a, void* stream,
                        const unsigned long long* seed) {
  if (!mod || !kernel || !a) return set_err(mod ? mod->ctx : nullptr, LCMX_ERR_ARGS, "launch: NULL argument");
  if (a->n_items <= 0 || a->n_tiles <= 0) return LCMX_OK;  // nothing to do
  if (!a->items || !a->tile_prefix || a->block <= 0 || a->block > 1024 || a->smem_bytes < 0)
    return set_err(mod->ctx, LCMX_ERR_ARGS, "launch: bad launch arguments");
  CUfunction f;
  int rc = get_func(mod, kernel, &f);
  if (rc) return rc;
  int per_sm = 0;
  {
    const auto key = std::make_tuple(f, a->block, a->smem_bytes);
    std::unique_lock<std::mutex> g(mod->mu);
    auto it = mod->geometry.find(key);
    if (it != mod->geometry.end()) {
      per_sm = it->second;
    } else {
      g.unlock();
      CUresult r = opt_in_smem(f, a->smem_bytes);
      if (r != CUDA_SUCCESS) return set_err(mod->ctx, LCMX_ERR_LAUNCH, "smem attribute: " + cu_msg(r));
      g_drv.OccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, a->block, (size_t)a->smem_bytes);
      if (per_sm < 1) per_sm = 1;
      g.lock();
      mod->geometry[key] = per_sm;
    }
  }
  int grid = a->grid;
  if (grid <= 0) grid = mod->ctx->sm_count * per_sm;
  if (grid > a->n_tiles) grid = a->n_tiles;
  const void* items = a->items;
  const int* prefix = a->tile_prefix;
  int n_items = a->n_items, n_tiles = a->n_tiles;
  unsigned long long s = seed ? *seed : 0ULL;
  void* params5[] = {(void*)&items, (void*)&prefix, (void*)&n_items, (void*)&n_tiles, (void*)&s};
  CUresult r = g_drv.LaunchKernel(f, (unsigned)grid, 1, 1, (unsigned)a->block, 1, 1, (unsigned)a->smem_bytes,
                              (CUstream)stream, params5, nullptr);
  if (r != CUDA_SUCCESS) return set_err(mod->ctx, LCMX_ERR_LAUNCH, std::string("launch ") + kernel + ": " + cu_msg(r));
  return LCMX_OK;
}

extern "C" int lcmx_module_status(lcmx_module* mod, const char* name, int* value, int reset) {
  if (!mod || !name || !value) return set_err(mod ? mod->ctx : nullptr, LCMX_ERR_ARGS, "lcmx_module_status: bad args");
  *value = 0;
  CUdeviceptr p = 0;
  size_t n = 0;
  CUresult r = g_drv.ModuleGetGlobal(&p, &n, mod->mod, name);
  if (r == CUDA_ERROR_NOT_FOUND) return LCMX_OK;  // the module has no such word: nothing to report
  if (r != CUDA_SUCCESS) return set_err(mod->ctx, LCMX_ERR_MODULE, std::string("status word ") + name + ": " + cu_msg(r));
  if (n < sizeof(int)) return set_err(mod->ctx, LCMX_ERR_MODULE, std::string("status word ") + name + " is too small");
  cudaError_t e = cudaMemcpy(value, reinterpret_cast<void*>(p), sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && reset && *value) e = cudaMemset(reinterpret_cast<void*>(p), 0, sizeof(int));
  if (e != cudaSuccess) return set_err(mod->ctx, LCMX_ERR_CUDA, std::string("status word: ") + cudaGetErrorString(e));
  return LCMX_OK;
}

extern "C" int lcmx_bellman_step(lcmx_module* mod, const char* kernel, const lcmx_launch_args* args, void* stream) {
  return launch_items(mod, kernel, args, stream, nullptr);
}

extern "C" int lcmx_expectation(lcmx_module* mod, const char* kernel, const lcmx_launch_args* args, void* stream) {
  return launch_items(mod, kernel, args, stream, nullptr);
}

extern "C" int lcmx_simulate(lcmx_module* mod, const char* kernel, const lcmx_launch_args* args,
                             unsigned long long seed, void* stream) {
  return launch_items(mod, kernel, args, stream, &seed);
}

extern "C" int lcmx_egm_step(lcmx_module* mod, const char* kernel, const lcmx_launch_args* args, void* stream) {
  return launch_items(mod, kernel, args, stream, nullptr);
}

// A list of item launches of generated kernels, issued in order on one
// stream: the per-launch host cost of a plan's step (hundreds of small
// launches) without a foreign-function call per launch.
extern "C" int lcmx_launch_list(const lcmx_launch_rec* recs, int n, void* stream) {
  if (n < 0 || (n > 0 && !recs)) return set_err(nullptr, LCMX_ERR_ARGS, "lcmx_launch_list: bad args");
  for (int i = 0; i < n; ++i) {
    const lcmx_launch_rec& r = recs[i];
    if (!r.module || !r.kernel) return set_err(nullptr, LCMX_ERR_ARGS, "lcmx_launch_list: record without a kernel");
    const int rc = launch_items(r.module, r.kernel, &r.args, stream, r.with_seed ? &r.seed : nullptr);
    if (rc) return rc;
  }
  return LCMX_OK;
}

// ------------------------------------------------------- non-finite count
__global__ void lcmx_nonfinite_kernel(const double* __restrict__ x, long long n, unsigned long long* counts) {
  unsigned long long nan = 0, inf = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double v = x[i];
    nan += (v != v);
    inf += (v == __longlong_as_double(0x7ff0000000000000LL)) || (v == -__longlong_as_double(0x7ff0000000000000LL));
  }
  for (int o = 16; o > 0; o >>= 1) {
    nan += __shfl_xor_sync(0xffffffffu, nan, o);
    inf += __shfl_xor_sync(0xffffffffu, inf, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (nan) atomicAdd(&counts[0], nan);
    if (inf) atomicAdd(&counts[1], inf);
  }
}

extern "C" int lcmx_count_nonfinite(lcmx_ctx* ctx, const double* x, long long n, unsigned long long* counts_dev,
                                    void* stream) {
  if (!ctx || (!x && n > 0) || !counts_dev || n < 0) return set_err(ctx, LCMX_ERR_ARGS, "lcmx_count_nonfinite: bad args");
  if (n == 0) return LCMX_OK;
  long long blocks = (n + 255) / 256;
  long long cap = (long long)ctx->sm_count * 8;
  if (blocks > cap) blocks = cap;
  lcmx_nonfinite_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(x, n, counts_dev);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(ctx, LCMX_ERR_LAUNCH, std::string("nonfinite: ") + cudaGetErrorString(e));
  return LCMX_OK;
}

extern "C" int lcmx_copy_rows_d2h(lcmx_ctx* ctx, void* dst, size_t dst_pitch, const void* src, size_t src_pitch,
                                  size_t row_bytes, size_t rows, void* stream) {
  if (!ctx || (rows > 0 && (!dst || !src)) || row_bytes > dst_pitch || row_bytes > src_pitch)
    return set_err(ctx, LCMX_ERR_ARGS, "lcmx_copy_rows_d2h: bad args");
  if (rows == 0 || row_bytes == 0) return LCMX_OK;
  cudaError_t e = cudaMemcpy2DAsync(dst, dst_pitch, src, src_pitch, row_bytes, rows, cudaMemcpyDeviceToHost,
                                    (cudaStream_t)stream);
  if (e != cudaSuccess) return set_err(ctx, LCMX_ERR_LAUNCH, std::string("copy_rows_d2h: ") + cudaGetErrorString(e));
  return LCMX_OK;
}

// error helper shared with the other translation units of this library
int lcmx_set_error_from(lcmx_ctx* ctx, int code, const std::string& msg) { return set_err(ctx, code, msg); }

// device ordinal of a context (for translation units that cannot see the struct)
int lcmx_ctx_device_of(const lcmx_ctx* ctx) { return ctx ? ctx->device : 0; }
