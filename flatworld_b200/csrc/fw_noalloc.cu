// fw_noalloc.cu -- fw_step_noalloc: the gather substep (element corner forces,
// then a per-node gather in ascending element order, boundary conditions and
// symplectic Euler) for callers that must not allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is off limits -- a real-time
// control loop, where cudaMalloc may block and synchronise the device at an
// unpredictable moment; a host application whose device memory is handed out
// by its own pool allocator under a fixed budget, so a library that allocates
// behind its back breaks the accounting; a plug-in that is loaded into such a
// process.  The context API (fw_create / fw_finalize) allocates its buffers, so
// those callers cannot use it.
//
// This entry point allocates nothing.  The caller passes every input and
// output as device memory it owns.  The only scratch -- one float2 per triangle
// corner, written by the element kernel and read by the node kernel -- lives in
// the file-scope array g_noalloc_corners below, whose size is fixed at build
// time (FW_NOALLOC_MAX_ELEMS triangles, 3 MiB).  Every GPU that loads the
// library holds that array until the process exits.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/fwb200.h"
#include "fw_device.cuh"

namespace {

// Scratch of fw_step_noalloc: three corner forces per triangle.  Each substep
// writes every corner it later reads, so nothing here has to start at zero.
// All calls share this one array; calls that overlap on the GPU (different
// streams, or host threads calling at once) race on it.
static __device__ __align__(256) float2 g_noalloc_corners[3 * FW_NOALLOC_MAX_ELEMS];

constexpr int kNaBlock = 256;
constexpr int kMaxDevices = 64;

std::mutex g_na_mutex;
float2* g_na_addr[kMaxDevices] = {nullptr};

__global__ void k_na_elements(int N, int E, const float2* __restrict__ x, const int32_t* __restrict__ conn,
                              const float4* __restrict__ jinv, const float4* __restrict__ emat,
                              float4* __restrict__ j2_state, const float2* __restrict__ j2_param,
                              float2* __restrict__ corners) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  const float4 mm = emat[e];
  fw::ElemMat m;
  m.area = mm.x;
  m.lam = mm.y;
  m.mu = mm.z;
  const int type = (int)mm.w;
  m.word = type & 3;
  const int n0 = conn[3 * e], n1 = conn[3 * e + 1], n2 = conn[3 * e + 2];
  // Only triangles (types 1-3) with node ids inside [0, N) are evaluated; any
  // other record (a spring, type 0, has no third node) adds no force and
  // reads nothing out of bounds.
  const bool valid = type >= 1 && type <= 3 && (unsigned)n0 < (unsigned)N && (unsigned)n1 < (unsigned)N &&
                     (unsigned)n2 < (unsigned)N;
  float2 f1 = make_float2(0.f, 0.f), f2 = f1, f3 = f1;
  if (valid) {
    const float2 a = x[n0], b = x[n1], c = x[n2];
    float4 j2 = make_float4(0.f, 0.f, 0.f, 0.f);
    // J2 triangles without state arrays never yield: an infinite yield stress
    // keeps the radial return off, so they respond with the elastic trial stress.
    float sy = __int_as_float(0x7f800000), H = 0.f;
    const bool mises = fw::elem_type(m.word) == fw::MAT_MISES && j2_state != nullptr;
    if (mises) {
      j2 = j2_state[e];
      sy = j2_param[e].x;
      H = j2_param[e].y;
    }
    fw::element_forces(a, b, c, jinv[e], m, sy, H, j2, f1, f2, f3);
    if (mises) j2_state[e] = j2;
  }
  corners[3 * e] = f1;
  corners[3 * e + 1] = f2;
  corners[3 * e + 2] = f3;
}

__global__ void k_na_nodes(int N, float2* __restrict__ x, float2* __restrict__ v,
                           const int32_t* __restrict__ node_bc, const float2* __restrict__ bc_values,
                           const float* __restrict__ mass, const int32_t* __restrict__ csr_off,
                           const int32_t* __restrict__ csr_slot, const float2* __restrict__ corners,
                           float dt, float damping) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  float2 f = make_float2(0.f, 0.f);
  for (int k = csr_off[i]; k < csr_off[i + 1]; ++k) {
    const float2 c = corners[csr_slot[k]];
    f.x += c.x;
    f.y += c.y;
  }
  float2 xi = x[i], vi = v[i];
  fw::integrate(node_bc[i] & 0x1FF, f, mass[i], bc_values[i], dt, damping, xi, vi);
  x[i] = xi;
  v[i] = vi;
}

int na_error(char* err, int32_t err_len, int code, const char* msg) {
  if (err && err_len > 0) snprintf(err, (size_t)err_len, "%s", msg);
  return code;
}

}  // namespace

extern "C" int fw_step_noalloc(int32_t n_nodes, int32_t n_elems, int32_t n_steps, float dt,
                               float damping, float* x, float* v, const int32_t* node_bc,
                               const float* bc_values, const float* mass, const int32_t* conn,
                               const float* jinv, const float* elem_mat, float* j2_state,
                               const float* j2_param, const int32_t* csr_off,
                               const int32_t* csr_slot, void* stream, char* err, int32_t err_len) {
  if (n_elems > FW_NOALLOC_MAX_ELEMS) {
    char msg[160];
    snprintf(msg, sizeof(msg), "fw_step_noalloc: %d triangles exceed the built-in scratch limit of %d",
             n_elems, FW_NOALLOC_MAX_ELEMS);
    return na_error(err, err_len, FW_ERR_ARG, msg);
  }
  if (n_nodes <= 0 || n_elems <= 0 || n_steps < 0)
    return na_error(err, err_len, FW_ERR_ARG, "fw_step_noalloc: need n_nodes > 0, n_elems > 0, n_steps >= 0");
  if (!x || !v || !node_bc || !bc_values || !mass || !conn || !jinv || !elem_mat || !csr_off || !csr_slot)
    return na_error(err, err_len, FW_ERR_ARG, "fw_step_noalloc: a required device pointer is NULL");
  if ((j2_state == nullptr) != (j2_param == nullptr))
    return na_error(err, err_len, FW_ERR_ARG,
                    "fw_step_noalloc: j2_state and j2_param must both be given or both be NULL");
  {
    // An error left by earlier work of the caller is reported as such, not as
    // a failure of this call's launches (and is left in place for the caller).
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) {
      char msg[200];
      snprintf(msg, sizeof(msg), "fw_step_noalloc: a CUDA error was pending before the call: %s",
               cudaGetErrorString(pending));
      return na_error(err, err_len, FW_ERR_CUDA, msg);
    }
  }
  // Set-up, once per device: the device address of the scratch array.  In host
  // code the array's name is a host-side stand-in, not a device address, so it
  // must be resolved with cudaGetSymbolAddress while that device is current.
  // The address is cached for the life of the process: after cudaDeviceReset
  // the module may be loaded elsewhere, so calls after a reset are unsupported.
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return na_error(err, err_len, FW_ERR_CUDA, "fw_step_noalloc: no current CUDA device");
  float2* corners = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_na_mutex);
    if (!g_na_addr[dev]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_corners);
      if (e != cudaSuccess || !p) {
        char msg[200];
        snprintf(msg, sizeof(msg), "fw_step_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        return na_error(err, err_len, FW_ERR_CUDA, msg);
      }
      g_na_addr[dev] = static_cast<float2*>(p);
    }
    corners = g_na_addr[dev];
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int ge = (n_elems + kNaBlock - 1) / kNaBlock, gn = (n_nodes + kNaBlock - 1) / kNaBlock;
  for (int k = 0; k < n_steps; ++k) {
    k_na_elements<<<ge, kNaBlock, 0, s>>>(n_nodes, n_elems, reinterpret_cast<const float2*>(x), conn,
                                          reinterpret_cast<const float4*>(jinv),
                                          reinterpret_cast<const float4*>(elem_mat),
                                          reinterpret_cast<float4*>(j2_state),
                                          reinterpret_cast<const float2*>(j2_param), corners);
    k_na_nodes<<<gn, kNaBlock, 0, s>>>(n_nodes, reinterpret_cast<float2*>(x), reinterpret_cast<float2*>(v),
                                       node_bc, reinterpret_cast<const float2*>(bc_values), mass, csr_off,
                                       csr_slot, corners, dt, damping);
    if (k == 0 || k == n_steps - 1) {  // launch errors: after the first pair, and at the end
      const cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) {
        char msg[200];
        snprintf(msg, sizeof(msg), "fw_step_noalloc: launch failed: %s", cudaGetErrorString(e));
        return na_error(err, err_len, FW_ERR_CUDA, msg);
      }
    }
  }
  return FW_OK;
}
