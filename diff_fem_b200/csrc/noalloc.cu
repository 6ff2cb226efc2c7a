// noalloc.cu — the corotated local step (J d of FEM tets) for callers that
// cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: code running inside a memory pool that
// owns every byte of the device heap, a host runtime that is only allowed to
// hand the library pre-allocated buffers, or code on a path where an
// allocation would stall other work on the GPU.  This entry point needs no
// allocation at all: the caller passes its inputs and outputs as device
// pointers, and the per-(tet, corner) scratch of the two-pass J d assembly
// lives in the file-scope array below, which every GPU that loads the library
// holds (DFEM_NOALLOC_MAX_TETS * 12 doubles, 6 MiB) until the process exits.
//
// The scratch is shared by every call on a device and keeps the last call's
// contents.  Each call writes every scratch entry it reads before reading it,
// so nothing has to start at zero; but calls that overlap on the GPU (two
// streams, or two host threads) race on it and must be serialised by the caller.
//
// Indices are checked on the device: a tet vertex outside [0, n_vertices) or
// an incidence slot outside [0, 4 n_tets) is skipped (no access is made through
// it), the affected output vertex is set to NaN, and a second file-scope word
// records the fault; the next call on the device reads that word first and
// returns DFEM_ERR_INVALID if it is set (then clears it).
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/dfem.h"
#include "pd_math.cuh"

namespace dfem {
namespace {

static __device__ __align__(256) double g_noalloc_slots[(size_t)DFEM_NOALLOC_MAX_TETS * 12];
static __device__ int g_noalloc_bad_index;  // 1: a call met an index out of range (see above)

constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_slots_addr[kMaxDevices] = {nullptr};  // device address of g_noalloc_slots per device

}  // namespace

int report_error(int code, const std::string& msg);  // engine.cu: sets dfem_last_error()

namespace {

int set_err(int code, const std::string& m) { return report_error(code, m); }

__global__ void k_noalloc_tets(int N, int T, const double* __restrict__ x, const int* __restrict__ tets,
                               const double* __restrict__ inv_dm, const double* __restrict__ w_rot,
                               const double* __restrict__ w_vol, double* __restrict__ slots) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  int vi[4];
  Vec3<double> xv[4];
  bool bad = false;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    vi[a] = tets[4 * t + a];
    bad = bad || vi[a] < 0 || vi[a] >= N;
  }
  if (bad) {  // skip the tet: its slots become NaN, which the gather passes on
    g_noalloc_bad_index = 1;
    for (int k = 0; k < 12; ++k) slots[12 * (size_t)t + k] = __longlong_as_double(0x7ff8000000000000LL);
    return;
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) xv[a] = mk3(x[3 * vi[a]], x[3 * vi[a] + 1], x[3 * vi[a] + 2]);
  // G[v][j]: F(:,j) = sum_v G[v][j] x_v, from invDm (row-major)
  double G[4][3];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    double a = inv_dm[9 * t + 0 + j], b = inv_dm[9 * t + 3 + j], c = inv_dm[9 * t + 6 + j];
    G[1][j] = a; G[2][j] = b; G[3][j] = c; G[0][j] = -(a + b + c);
  }
  Mat3<double> F, md, mdv;
#pragma unroll
  for (int j = 0; j < 3; ++j) F.c[j] = G[0][j] * xv[0] + G[1][j] * xv[1] + G[2][j] * xv[2] + G[3][j] * xv[3];
  corot_project(F, md, mdv);
  double wr = w_rot[t], wv = w_vol[t];
  Vec3<double> P[3];
#pragma unroll
  for (int j = 0; j < 3; ++j) P[j] = wr * md.c[j] + wv * mdv.c[j];
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    Vec3<double> f = G[a][0] * P[0] + G[a][1] * P[1] + G[a][2] * P[2];
    double* o = slots + 12 * (size_t)t + 3 * a;
    o[0] = f.x; o[1] = f.y; o[2] = f.z;
  }
}

__global__ void k_noalloc_gather(int N, int T, const int* __restrict__ vtx_ptr, const int* __restrict__ vtx_slot,
                                 const double* __restrict__ slots, double* __restrict__ out) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  double a0 = 0, a1 = 0, a2 = 0;
  const int k0 = vtx_ptr[i], k1 = vtx_ptr[i + 1];
  bool bad = k0 < 0 || k1 < k0 || k1 > 4 * T;
  for (int k = k0; !bad && k < k1; ++k) {
    const int sl = vtx_slot[k];
    if (sl < 0 || sl >= 4 * T) { bad = true; break; }
    const double* q = slots + 3 * (size_t)sl;
    a0 += q[0]; a1 += q[1]; a2 += q[2];
  }
  if (bad) {
    g_noalloc_bad_index = 1;
    a0 = a1 = a2 = __longlong_as_double(0x7ff8000000000000LL);
  }
  out[3 * i] = a0; out[3 * i + 1] = a1; out[3 * i + 2] = a2;
}

}  // namespace
}  // namespace dfem

using namespace dfem;

extern "C" int dfem_eval_corotated_noalloc(int32_t n_vertices, int32_t n_tets, const double* x, const int32_t* tets,
                                           const double* inv_dm, const double* w_rot, const double* w_vol,
                                           const int32_t* vtx_ptr, const int32_t* vtx_slot, double* jd_out,
                                           void* stream) {
  if (n_vertices < 0 || n_tets < 0) return set_err(DFEM_ERR_INVALID, "negative size");
  if (n_tets > DFEM_NOALLOC_MAX_TETS)
    return set_err(DFEM_ERR_INVALID, "dfem_eval_corotated_noalloc: n_tets = " + std::to_string(n_tets) +
                                         " exceeds the static scratch limit DFEM_NOALLOC_MAX_TETS = " +
                                         std::to_string(DFEM_NOALLOC_MAX_TETS));
  if (n_vertices == 0) return DFEM_OK;
  if (!x || !jd_out || !vtx_ptr || (n_tets > 0 && (!tets || !inv_dm || !w_rot || !w_vol || !vtx_slot)))
    return set_err(DFEM_ERR_INVALID, "null pointer argument");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_err(DFEM_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return set_err(DFEM_ERR_INVALID, "device index beyond the per-device table");
  double* slots = nullptr;
  {
    // first call on this device: look up the device address of the static
    // scratch (host code may not use the array's name as a device pointer)
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_slots_addr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_slots);
      if (e != cudaSuccess) return set_err(DFEM_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_slots_addr[dev] = static_cast<double*>(p);
    }
    slots = g_slots_addr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  {
    // an earlier call on this device met an index out of range: report it once
    // (this waits for the work already queued on `stream`)
    int bad = 0;
    e = cudaMemcpyFromSymbolAsync(&bad, g_noalloc_bad_index, sizeof(int), 0, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_err(DFEM_ERR_CUDA, cudaGetErrorString(e));
    if (bad) {
      const int zero = 0;
      e = cudaMemcpyToSymbolAsync(g_noalloc_bad_index, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, s);
      if (e == cudaSuccess) e = cudaStreamSynchronize(s);
      if (e != cudaSuccess) return set_err(DFEM_ERR_CUDA, cudaGetErrorString(e));
      return set_err(DFEM_ERR_INVALID, "dfem_eval_corotated_noalloc: an earlier call met a vertex index or incidence "
                                       "slot out of range (its outputs were NaN)");
    }
  }
  if (n_tets > 0)
    k_noalloc_tets<<<(n_tets + 127) / 128, 128, 0, s>>>(n_vertices, n_tets, x, tets, inv_dm, w_rot, w_vol, slots);
  k_noalloc_gather<<<(n_vertices + 127) / 128, 128, 0, s>>>(n_vertices, n_tets, vtx_ptr, vtx_slot, slots, jd_out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return set_err(DFEM_ERR_CUDA, cudaGetErrorString(e));
  return DFEM_OK;
}
