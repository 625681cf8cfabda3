// Leader kernel: the serial part of one mCDFCI iteration, run by one CTA of
// 512 threads between two column-kernel launches (its device code is in
// leader_body.cuh).
//
//   finish iteration t-1   z[D_c] = new_z_c for the picked D_c (the exact
//                          recompute that overwrites the accumulated z,
//                          src/wavefunction.h:557-565); xz += sum_c dot_c
//                          (src/wavefunction.h:583); occupancy check
//                          (src/wavefunction.h:594-599)
//   refetch                (x, z) of every column's candidates from the table
//                          (src/wavefunction.h:567-575)
//   pick                   the k distinct determinants with the largest
//                          |x*xx*scale^2 + z|, ties to the larger determinant
//                          in the reference order (CoordinatePickGcdGrad,
//                          src/solver.h:118-143,196-224)
//   H_sub                  k x k sub-matrix (CDFCI::get_hamiltonian_submatrix,
//                          src/solver.h:637-670): upper triangle from
//                          get_off_diagonal(det_i, det_j) for i < j, diagonal
//                          from get_diagonal (src/hamiltonian.h:252-328)
//   eig update             dx, scale and xx (CoordinateUpdateEig,
//                          src/solver.h:333-609)
//   update_x               x[D_c] += dx_c, xz += z[D_c] * dx_c
//                          (WaveFunctionCuckoo::update_x, src/wavefunction.h:425-451)
//   publish                the k picked determinants, dx, H_cc, xx*scale^2
//                          and scale for the column kernel.
#include <mutex>

#include "leader_body.cuh"

namespace mcd {
namespace {

__global__ void __launch_bounds__(kLT, 1) leader_kernel(LeaderLaunch L) { leader_body(L); }

// One CTA per instance of a batch.
__global__ void __launch_bounds__(kLT, 1) leader_kernel_batch(LeaderBatch B) { leader_body(B.L[blockIdx.x]); }

// Initial state (CDFCI::solve, src/solver.h:862-873): x = e_ref, z = H[:,ref]
// through one column update with dx = 1, xx = scale = 1, xz = 0.
__global__ void init_kernel(LeaderLaunch L, Det ref, double ref_diag) {
  IterState* S = L.st;
  bool inserted = false;
  const long long slot = table_upsert(L.tab, ref.a, ref.b, inserted);
  if (slot < 0) {
    S->k_cur = 0;
    return;
  }
  Slot* sp = L.tab.slots + slot;
  const double x0 = sp->x;
  sp->x = x0 + 1.0;
  S->x_size = (x0 == 0.0) ? 1 : 0;
  S->xx = dd{1.0, 0.0};
  S->scale = dd{1.0, 0.0};
  S->xz = dd_add_d(dd{0.0, 0.0}, sp->z * 1.0);
  S->xss = dd{1.0, 0.0};
  S->k_cur = 1;
  S->det[0] = ref;
  S->slot[0] = slot;
  S->dx[0] = 1.0;
  S->hdiag[0] = ref_diag;
  S->emitted = 0;
  S->updates = 0;
  S->z_size = 0;
  S->iter = 0;
  S->dx_max = 1.0;
  S->eig_residual_max = 0.0;
  S->last_branch = 0;
  S->pending = 1;
}

__global__ void debug_hsub_kernel(HamDev h, const Det* dets, int k, double* H) {
  __shared__ unsigned char s_occ[kLW][128];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int t = tid; t < k * k; t += blockDim.x) {
    const int i = t / k, j = t - i * k;
    if (i != j) H[t] = off_diagonal(h, dets[i], dets[j]);
  }
  for (int i = warp; i < k; i += blockDim.x / 32) {
    const double v = diagonal_warp(h, dets[i], s_occ[warp]);
    if (lane == 0) H[i * k + i] = v;
  }
}

// Lower triangle of the row-major k x k matrix H := its upper triangle (the
// part of H_sub the reference's dsyevr/dsymv calls read); block-wide.
__device__ void symmetrise_from_upper(double* H, int k) {
  for (int idx = threadIdx.x; idx < k * k; idx += blockDim.x) {
    const int i = idx / k, j = idx - i * k;
    if (i < j) H[j * k + i] = H[idx];
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kLT, 1) debug_eig_kernel(int k, double* H, const double* x, const double* z,
                                                           dd xx, dd xz, double* dx, dd* out, int* branch,
                                                           unsigned* err, double drop, int method, int* steps) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double s_x[kMaxK], s_z[kMaxK], s_dx[kMaxK];
  for (int i = threadIdx.x; i < k; i += blockDim.x) {
    s_x[i] = x[i];
    s_z[i] = z[i];
  }
  symmetrise_from_upper(H, k);
  SectionClock clk{nullptr, 0};
  const EigResult er =
      eig_update(H, k, s_x, s_z, xx, xz, s_dx, reinterpret_cast<double*>(smem), clk, drop, method);
  for (int i = threadIdx.x; i < k; i += blockDim.x) dx[i] = s_dx[i];
  if (threadIdx.x == 0) {
    out[0] = er.xx;
    out[1] = er.scale;
    *branch = er.branch;
    *err = er.ok ? 0u : kErrEig;
    if (steps) *steps = er.shift_steps;
  }
}

}  // namespace

size_t leader_smem_bytes(int k, int m) {
  size_t P = 2;
  while (P < static_cast<size_t>(k) * m) P <<= 1;
  const size_t pick = P * 4 + 2 * P * 4;  // slots + hash set (the hash set area later holds P doubles)
  const size_t hs = (k <= 64 ? static_cast<size_t>(k) * k : 0) * sizeof(double);
  const size_t eig = hs + eig_work_doubles(k) * sizeof(double);
  return pick > eig ? pick : eig;
}

namespace {

// The dynamic shared-memory limit of a kernel is a per-device attribute:
// each device's largest configured size is kept, and the attribute is set
// (outside stream capture: the first launch on a device precedes it) when a
// launch on the current device needs more.
constexpr int kMaxDevices = 64;
struct SmemLimit {
  std::mutex mu;
  size_t bytes[kMaxDevices] = {};
};

cudaError_t ensure_smem(const void* func, size_t bytes, SmemLimit& lim) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(lim.mu);
  if (bytes <= lim.bytes[dev]) return cudaSuccess;
  e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes));
  if (e == cudaSuccess) lim.bytes[dev] = bytes;
  return e;
}

SmemLimit g_leader_smem, g_leader_batch_smem;

}  // namespace

cudaError_t prepare_leader(const LeaderLaunch& a) {
  return ensure_smem(reinterpret_cast<const void*>(leader_kernel), leader_smem_bytes(a.k_req, a.m), g_leader_smem);
}

cudaError_t launch_leader(const LeaderLaunch& a, cudaStream_t s) {
  const size_t bytes = leader_smem_bytes(a.k_req, a.m);
  cudaError_t e = ensure_smem(reinterpret_cast<const void*>(leader_kernel), bytes, g_leader_smem);
  if (e != cudaSuccess) return e;
  leader_kernel<<<1, kLT, bytes, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_leader_batch(const LeaderBatch& b, cudaStream_t s) {
  if (b.n < 1 || b.n > kMaxBatch) return cudaErrorInvalidValue;
  const size_t bytes = leader_smem_bytes(b.L[0].k_req, b.L[0].m);
  cudaError_t e = ensure_smem(reinterpret_cast<const void*>(leader_kernel_batch), bytes, g_leader_batch_smem);
  if (e != cudaSuccess) return e;
  leader_kernel_batch<<<b.n, kLT, bytes, s>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_init(const LeaderLaunch& a, Det hf, double hf_diag, cudaStream_t s) {
  init_kernel<<<1, 1, 0, s>>>(a, hf, hf_diag);
  return cudaGetLastError();
}

cudaError_t launch_finish(const LeaderLaunch& a, cudaStream_t s) {
  finish_kernel<<<1, kMaxK, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t debug_hsub(const HamDev& h, const Det* dets, int k, double* hsub, cudaStream_t s) {
  debug_hsub_kernel<<<1, 256, 0, s>>>(h, dets, k, hsub);
  return cudaGetLastError();
}

cudaError_t debug_eig(int k, double* hsub, const double* x, const double* z, dd xx, dd xz, double* dx,
                      dd* new_xx_scale, int* branch, unsigned* err, cudaStream_t s, double drop, int* steps,
                      int method) {
  const size_t bytes = eig_work_doubles(k) * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(debug_eig_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       static_cast<int>(bytes));
  if (e != cudaSuccess) return e;
  debug_eig_kernel<<<1, kLT, bytes, s>>>(k, hsub, x, z, xx, xz, dx, new_xx_scale, branch, err, drop, method, steps);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// eig_update_static: the eig update of debug_eig run on a file-scope device
// array instead of cudaMalloc'd buffers.  Layout in doubles: H [kStaticEigMaxK^2],
// x, z, dx [kStaticEigMaxK each], new xx and scale as two dd, then one word
// holding the branch (int) and the error word (unsigned).  static_eig_kernel
// writes dx[0..k), both dd, the branch and the error word on every launch, so
// no part of the array has to start at zero or be cleared between calls.

namespace {

constexpr size_t kStaticEigH = 0;
constexpr size_t kStaticEigX = kStaticEigH + static_cast<size_t>(kStaticEigMaxK) * kStaticEigMaxK;
constexpr size_t kStaticEigZ = kStaticEigX + kStaticEigMaxK;
constexpr size_t kStaticEigDx = kStaticEigZ + kStaticEigMaxK;
constexpr size_t kStaticEigOut = kStaticEigDx + kStaticEigMaxK;  // 2 dd = 4 doubles
constexpr size_t kStaticEigFlags = kStaticEigOut + 4;            // int branch, unsigned err
constexpr size_t kStaticEigDoubles = kStaticEigFlags + 1;

static __device__ __align__(256) double g_static_eig_scratch[kStaticEigDoubles];

// debug_eig_kernel on the array at `base` (the address of
// g_static_eig_scratch on this device).  A kernel of its own, so that its
// shared-memory attribute, set once per device, is not changed by debug_eig.
__global__ void __launch_bounds__(kLT, 1) static_eig_kernel(int k, double* base, dd xx, dd xz) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double s_x[kMaxK], s_z[kMaxK], s_dx[kMaxK];
  for (int i = threadIdx.x; i < k; i += blockDim.x) {
    s_x[i] = base[kStaticEigX + i];
    s_z[i] = base[kStaticEigZ + i];
  }
  symmetrise_from_upper(base + kStaticEigH, k);
  SectionClock clk{nullptr, 0};
  const EigResult er =
      eig_update(base + kStaticEigH, k, s_x, s_z, xx, xz, s_dx, reinterpret_cast<double*>(smem), clk, 0.0, 0);
  for (int i = threadIdx.x; i < k; i += blockDim.x) base[kStaticEigDx + i] = s_dx[i];
  if (threadIdx.x == 0) {
    dd* out = reinterpret_cast<dd*>(base + kStaticEigOut);
    out[0] = er.xx;
    out[1] = er.scale;
    int* flags = reinterpret_cast<int*>(base + kStaticEigFlags);
    flags[0] = er.branch;
    flags[1] = er.ok ? 0 : static_cast<int>(kErrEig);
  }
}

// Set-up, with the device current: the address of the array in this
// device's copy of the module, and the kernel's shared-memory attribute for
// the largest k.  Both are looked up on every call (neither allocates, and
// after the first call on a device the module is loaded, so they are cheap),
// so that no address outlives the context it belongs to (a cudaDeviceReset
// between two calls gives the second a fresh one).
cudaError_t static_eig_setup(double** base) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_static_eig_scratch);
  if (e != cudaSuccess) return e;
  e = cudaFuncSetAttribute(static_eig_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           static_cast<int>(eig_work_doubles(kStaticEigMaxK) * sizeof(double)));
  if (e != cudaSuccess) return e;
  *base = static_cast<double*>(p);
  return cudaSuccess;
}

}  // namespace

cudaError_t eig_update_static(int k, const double* hsub, const double* x, const double* z, dd xx, dd xz,
                              double* dx, dd* new_xx_scale, int* branch, unsigned* err, cudaStream_t s) {
  if (k < 1 || k > kStaticEigMaxK) return cudaErrorInvalidValue;  // the caller reports the limit
  double* base = nullptr;
  cudaError_t e = static_eig_setup(&base);
  if (e != cudaSuccess) return e;
  double* dH = base + kStaticEigH;
  double* dX = base + kStaticEigX;
  double* dZ = base + kStaticEigZ;
  double* dDx = base + kStaticEigDx;
  dd* dOut = reinterpret_cast<dd*>(base + kStaticEigOut);
  int* dBranch = reinterpret_cast<int*>(base + kStaticEigFlags);
  unsigned* dErr = reinterpret_cast<unsigned*>(dBranch + 1);
  const size_t kk = static_cast<size_t>(k);
  if ((e = cudaMemcpyAsync(dH, hsub, sizeof(double) * kk * kk, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(dX, x, sizeof(double) * kk, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(dZ, z, sizeof(double) * kk, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
  static_eig_kernel<<<1, kLT, eig_work_doubles(k) * sizeof(double), s>>>(k, base, xx, xz);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(dx, dDx, sizeof(double) * kk, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(new_xx_scale, dOut, sizeof(dd) * 2, cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(branch, dBranch, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
  if ((e = cudaMemcpyAsync(err, dErr, sizeof(unsigned), cudaMemcpyDeviceToHost, s)) != cudaSuccess) return e;
  return cudaStreamSynchronize(s);
}

}  // namespace mcd
