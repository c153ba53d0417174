// Error reporting, per-device one-time set-up and small C-ABI utilities.
#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <set>
#include <string>
#include <utility>

#include "n3_common.cuh"

namespace n3host {

static thread_local std::string g_last_error;

int set_error(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int check_launch(const char* what) {
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return set_error(N3_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  return N3_OK;
}

int build_dir_lut(cudaStream_t st);  // score.cu

static std::mutex g_init_mutex;
static bool g_tables_ready[64];
static int g_sm_count[64];

static int current_device(int* dev) {
  const cudaError_t e = cudaGetDevice(dev);
  if (e != cudaSuccess) return set_error(N3_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (*dev < 0 || *dev >= 64) return set_error(N3_ERR_CUDA, "device ordinal %d unsupported", *dev);
  return N3_OK;
}

// One-time, per-device construction of the device-resident lookup tables
// (the gcd-reduced direction table used by the slope kernels).  Runs on a
// private stream and waits for it, so the first call on a device must not be
// made while a stream is being captured into a CUDA graph.
int ensure_device_tables() {
  int dev = 0;
  N3_TRY(current_device(&dev));
  std::lock_guard<std::mutex> lock(g_init_mutex);
  if (g_tables_ready[dev]) return N3_OK;
  cudaStream_t st;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return check_launch("cudaStreamCreate");
  int rc = build_dir_lut(st);
  const cudaError_t e = cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  if (rc != N3_OK) return rc;
  if (e != cudaSuccess) return set_error(N3_ERR_CUDA, "table set-up: %s", cudaGetErrorString(e));
  g_tables_ready[dev] = true;
  return N3_OK;
}

// Opts `kernel` into `bytes` of dynamic shared memory, once per (kernel, device).
int allow_smem(const void* kernel, size_t bytes) {
  static std::mutex mu;
  static std::set<std::pair<const void*, int>> done;
  int dev = 0;
  N3_TRY(current_device(&dev));
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_pair(kernel, dev);
  if (done.count(key)) return N3_OK;
  const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return set_error(N3_ERR_CUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
  done.insert(key);
  return N3_OK;
}

int sm_count() {
  int dev = 0;
  if (current_device(&dev) != N3_OK) return 148;
  if (g_sm_count[dev] == 0) {
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) v = 148;
    g_sm_count[dev] = v;
  }
  return g_sm_count[dev];
}

}  // namespace n3host

namespace n3host {
int prepare_score();
int prepare_delta();
int prepare_tempering();
int prepare_mlp();
}  // namespace n3host

extern "C" {

int n3_version(void) { return 100; }

int n3_init_device(void) {
  N3_TRY(n3host::ensure_device_tables());
  N3_TRY(n3host::prepare_score());
  N3_TRY(n3host::prepare_delta());
  N3_TRY(n3host::prepare_tempering());
  return n3host::prepare_mlp();
}

const char* n3_last_error(void) { return n3host::g_last_error.c_str(); }

}  // extern "C"

// ---------------------------------------------------------------------------
// CUDA graphs: capture a fixed sequence of launches once, replay it cheaply.
// ---------------------------------------------------------------------------
extern "C" {

int n3_graph_begin(void* stream) {
  if (stream == nullptr) return n3host::set_error(N3_ERR_ARG, "graph capture needs a non-default stream");
  const cudaError_t e = cudaStreamBeginCapture((cudaStream_t)stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return n3host::set_error(N3_ERR_CUDA, "cudaStreamBeginCapture: %s", cudaGetErrorString(e));
  return N3_OK;
}

int n3_graph_end(void* stream, void** graph_exec) {
  if (graph_exec == nullptr) return n3host::set_error(N3_ERR_ARG, "null graph handle");
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture((cudaStream_t)stream, &g);
  if (e != cudaSuccess) return n3host::set_error(N3_ERR_CUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(e));
  cudaGraphExec_t x = nullptr;
  e = cudaGraphInstantiate(&x, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) return n3host::set_error(N3_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
  *graph_exec = (void*)x;
  return N3_OK;
}

int n3_graph_launch(void* graph_exec, void* stream) {
  if (graph_exec == nullptr) return n3host::set_error(N3_ERR_ARG, "null graph handle");
  const cudaError_t e = cudaGraphLaunch((cudaGraphExec_t)graph_exec, (cudaStream_t)stream);
  if (e != cudaSuccess) return n3host::set_error(N3_ERR_CUDA, "cudaGraphLaunch: %s", cudaGetErrorString(e));
  return N3_OK;
}

int n3_graph_destroy(void* graph_exec) {
  if (graph_exec != nullptr) cudaGraphExecDestroy((cudaGraphExec_t)graph_exec);
  return N3_OK;
}

}  // extern "C"
