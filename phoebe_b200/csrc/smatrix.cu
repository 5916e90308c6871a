// Scattering matrix in device memory and the matrix-vector products of the
// builder's matrix modes.
//
//   * ScatteringMatrix::dot / offDiagonalDot of a stored matrix
//     (src/bte/scattering.cpp:180-265, 266-330), for the matrix that
//     PhScatteringMatrix::builder builds with switchCase 0;
//   * the product with the rate slabs of one q2 chunk, which is how the
//     builder's switchCase 1 (src/bte/ph_scattering.cpp:408-431, 549-572) runs
//     here: A x without storing A, chunk by chunk.
//
// Both are reads of FP64 matrix blocks once each, bound by HBM bandwidth: one
// thread per row (coalesced down a column), a block of columns per CTA with
// their x values staged in shared memory, and one atomic add per row and
// vector component at the end.  One input vector (the iterative solvers'
// case) has its own instantiation, whose 3 accumulators leave room for 8
// loads in flight per thread; more vectors go 4 per pass.
#include <cusolverDn.h>
#include <cusolverMg.h>
#include <dlfcn.h>

#include <type_traits>

#include <algorithm>
#include <cstdlib>
#include <cstring>

#include "pair_common.cuh"
#include "phx_consts.h"
#include "phx_internal.h"

using pairc::mesh_neg;

namespace {

constexpr int kDotRows = 256;   // rows (threads) per CTA
constexpr int kDotVec = 4;      // input vectors per pass (several vectors)

template <int NV>
__global__ void __launch_bounds__(kDotRows) smatrix_dot_kernel(phx_dot_args A, int cols_per_block) {
  constexpr int kDotV3 = 3 * NV;
  extern __shared__ __align__(16) double dsm[];
  double* xp = dsm;                                  // [cols][kDotV3]
  double* xm = xp + (size_t)cols_per_block * kDotV3; // [cols][kDotV3] (slabs)
  int* stp = reinterpret_cast<int*>(xm + (A.Sm ? (size_t)cols_per_block * kDotV3 : 0));
  int* stm = stp + cols_per_block;
  const int c = blockIdx.z % A.nT, v0 = (blockIdx.z / A.nT) * NV;
  const int nv = min(NV, A.nvec - v0);
  const int k0 = blockIdx.y * cols_per_block, kn = min(cols_per_block, A.ncols - k0);
  for (int t = threadIdx.x; t < cols_per_block; t += blockDim.x) {
    int sp = 0, sm = 0;
    if (t < kn) {
      const int k = k0 + t;
      if (A.slab) {
        const int j = k / A.nb, b2 = k - j * A.nb, iq2 = A.q2_first + j;
        sp = iq2 * A.nb + b2;
        sm = mesh_neg(iq2, A.n0, A.n1, A.n2) * A.nb + b2;
      } else {
        sp = k;
      }
    }
    stp[t] = sp;
    stm[t] = sm;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < cols_per_block * kDotV3; e += blockDim.x) {
    const int t = e / kDotV3, vi = e - t * kDotV3, v = vi / 3, i = vi - 3 * v;
    double a = 0.0, b = 0.0;
    if (t < kn && v < nv) {
      const double* xv = A.x + (((size_t)(v0 + v) * A.nT + c) * 3 + i) * A.ns;
      a = xv[stp[t]];
      if (A.Sm) b = xv[stm[t]];
      if (A.skip == 1 && A.E[stp[t]] < phxc::phExcludeCutoff) a = 0.0;
    }
    xp[e] = a;
    if (A.Sm) xm[e] = b;
  }
  __syncthreads();
  const int r = blockIdx.x * kDotRows + threadIdx.x;
  if (r >= A.ns) return;
  if (A.skip == 1 && A.E[r] < phxc::phExcludeCutoff) return;
  double acc[kDotV3];
#pragma unroll
  for (int vi = 0; vi < kDotV3; ++vi) acc[vi] = 0.0;
  const double* P = A.Sp + c * A.tstride + (size_t)k0 * A.ld + r;
  if (A.Sm) {
    const double* Q = A.Sm + c * A.tstride + (size_t)k0 * A.ld + r;
#pragma unroll 4
    for (int t = 0; t < kn; ++t) {
      double a = __ldcs(P + (size_t)t * A.ld), b = __ldcs(Q + (size_t)t * A.ld);
      if (r == stp[t]) a = 0.0;
      if (r == stm[t]) b = 0.0;
#pragma unroll
      for (int vi = 0; vi < kDotV3; ++vi) acc[vi] += a * xp[t * kDotV3 + vi] - b * xm[t * kDotV3 + vi];
    }
  } else {
#pragma unroll 8
    for (int t = 0; t < kn; ++t) {
      double a = __ldcs(P + (size_t)t * A.ld);
      if (A.skip == 0 && r == stp[t]) a = 0.0;
#pragma unroll
      for (int vi = 0; vi < kDotV3; ++vi) acc[vi] += a * xp[t * kDotV3 + vi];
    }
  }
  for (int v = 0; v < nv; ++v)
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double s = acc[3 * v + i];
      if (s != 0.0) atomicAdd(A.y + (((size_t)(v0 + v) * A.nT + c) * 3 + i) * A.ns + r, s);
    }
}

__global__ void diag_term_kernel(int ns, int nT, int nvec, const double* __restrict__ lw,
                                 const double* __restrict__ x, double* __restrict__ y, const double* __restrict__ E,
                                 int finalize) {
  const size_t n = (size_t)nvec * nT * 3 * ns;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int s = (int)(e % ns);
    const int c = (int)((e / ns / 3) % nT);
    if (finalize && E[s] < phxc::phExcludeCutoff) y[e] = 0.0;
    else y[e] += lw[(size_t)c * ns + s] * x[e];
  }
}

__global__ void set_diag_kernel(int ns, long long ld, const double* __restrict__ diag, double* __restrict__ A) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < ns) A[(size_t)s * ld + s] = diag[s];
}

// out (nrows, ns) row-major = rows row0.. of the column-major A, through 32x32 tiles
__global__ void rows_kernel(int ns, long long ld, const double* __restrict__ A, int row0, int nrows,
                            double* __restrict__ out) {
  __shared__ double tile[32][33];
  const int cb = blockIdx.x * 32, rb = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int col = cb + k, r = rb + threadIdx.x;
    tile[k][threadIdx.x] = (col < ns && r < nrows) ? A[(size_t)col * ld + row0 + r] : 0.0;
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = rb + k, col = cb + threadIdx.x;
    if (r < nrows && col < ns) out[(size_t)r * ns + col] = tile[threadIdx.x][k];
  }
}

}  // namespace

namespace {

template <int NV>
int dot_launch(const phx_dot_args& a, cudaStream_t st) {
  // slabs: two blocks of columns per CTA; a stored matrix: one, longer
  const int cols = a.Sm ? 64 : 256;
  const size_t smem = sizeof(double) * cols * 3 * NV * (a.Sm ? 2 : 1) + sizeof(int) * 2 * cols;
  dim3 grid((a.ns + kDotRows - 1) / kDotRows, (a.ncols + cols - 1) / cols, a.nT * ((a.nvec + NV - 1) / NV));
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(smatrix_dot_kernel<NV>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  smatrix_dot_kernel<NV><<<grid, kDotRows, smem, st>>>(a, cols);
  return cudaGetLastError() == cudaSuccess ? PHX_OK : PHX_ERR_CUDA;
}

// (A + A^T) / 2 in place (SerialMatrix::symmetrize, src/algebra/SMatrix.cpp:124-138):
// the CTA of tile pair (ti, tj), ti <= tj, stages both 32 x 32 tiles in shared memory
__global__ void symmetrize_kernel(int ns, long long ld, double* __restrict__ A) {
  const int ti = blockIdx.y, tj = blockIdx.x;
  if (ti > tj) return;
  __shared__ double a[32][33], b[32][33];
  const int r0 = ti * 32, c0 = tj * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = r0 + threadIdx.x, c = c0 + k;        // a[k][x] = A(r0 + x, c0 + k)
    a[k][threadIdx.x] = (r < ns && c < ns) ? A[(size_t)c * ld + r] : 0.0;
    const int r2 = c0 + threadIdx.x, c2 = r0 + k;      // b[k][x] = A(c0 + x, r0 + k)
    b[k][threadIdx.x] = (r2 < ns && c2 < ns) ? A[(size_t)c2 * ld + r2] : 0.0;
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    // A(r0 + x, c0 + k) and A(c0 + k, r0 + x) both become their mean
    const double m = 0.5 * (a[k][threadIdx.x] + b[threadIdx.x][k]);
    const int r = r0 + threadIdx.x, c = c0 + k;
    if (r < ns && c < ns) A[(size_t)c * ld + r] = m;
  }
  if (ti == tj) return;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const double m = 0.5 * (b[k][threadIdx.x] + a[threadIdx.x][k]);
    const int r2 = c0 + threadIdx.x, c2 = r0 + k;
    if (r2 < ns && c2 < ns) A[(size_t)c2 * ld + r2] = m;
  }
}

// n(n+1) of each state at temperature T (Particle::getPopPopPm1 for phonons,
// src/particle.cpp), 0 for the excluded states (E < 0.1 cm^-1)
__global__ void poppm1_kernel(int ns, const double* __restrict__ E, double T, double* __restrict__ term) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= ns) return;
  const double e = E[s];
  if (e < phxc::phExcludeCutoff) {
    term[s] = 0.0;
    return;
  }
  const double x = sinh(e / (2.0 * T));
  term[s] = 0.25 / (x * x);
}

// ScatteringMatrix::a2Omega (src/bte/scattering.cpp:366-434): A(i, j) /=
// sqrt(n_i(n_i+1) n_j(n_j+1)) unless i or j is excluded, and the diagonal
// (the linewidths) /= n_i(n_i+1).  Threads down a column (coalesced), CTAs
// over row blocks x a stride of columns.
__global__ void __launch_bounds__(256) a2omega_kernel(int ns, long long ld, const double* __restrict__ term,
                                                       double* __restrict__ A, double* __restrict__ diag) {
  const int r = blockIdx.x * 256 + threadIdx.x;
  if (r >= ns) return;
  const double tr = term[r];
  if (blockIdx.y == 0 && tr != 0.0) diag[r] /= tr;
  if (tr == 0.0) return;
  for (int c = blockIdx.y; c < ns; c += gridDim.y) {
    const double tc = term[c];
    if (tc != 0.0) A[(size_t)c * ld + r] /= sqrt(tr * tc);
  }
}

// The relaxon populations of calcFromRelaxons (src/observable/
// phonon_thermal_cond.cpp:316-347): r(v, i, a) = g_a sum_s Theta(s, a) x(v, i, s),
// g_a = 1/lambda_a for lambda_a > 0, else 0.  One CTA per eigenvector a (a
// coalesced read of its column), x (nvec, 3, ns) from L2.
__global__ void __launch_bounds__(256) relaxon_project_kernel(int ns, long long ld, const double* __restrict__ Th,
                                                               const double* __restrict__ W, int nvec,
                                                               const double* __restrict__ x, double* __restrict__ r) {
  const int a = blockIdx.x;
  const double lam = W[a];
  const double* col = Th + (size_t)a * ld;
  __shared__ double red[8][3];
  for (int v = 0; v < nvec; ++v) {
    const double* xv = x + (size_t)v * 3 * ns;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0;
    for (int s = threadIdx.x; s < ns; s += 256) {
      const double t = col[s];
      s0 += t * xv[s];
      s1 += t * xv[ns + s];
      s2 += t * xv[2 * ns + s];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s0 += __shfl_xor_sync(0xffffffffu, s0, o);
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
      red[w][0] = s0;
      red[w][1] = s1;
      red[w][2] = s2;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
      double t = 0.0;
      for (int k = 0; k < 8; ++k) t += red[k][threadIdx.x];
      r[((size_t)v * 3 + threadIdx.x) * ns + a] = lam > 0.0 ? t / lam : 0.0;
    }
    __syncthreads();
  }
}

// A(c, r) = A(r, c) for r < c: the upper triangle copied onto the lower one
// (32 x 32 tiles of the upper triangle, one block each)
__global__ void mirror_upper_kernel(int ns, long long ld, double* __restrict__ A) {
  const int ti = blockIdx.y, tj = blockIdx.x;
  if (ti > tj) return;
  __shared__ double a[32][33];
  const int r0 = ti * 32, c0 = tj * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = r0 + threadIdx.x, c = c0 + k;   // a[k][x] = A(r0 + x, c0 + k)
    a[k][threadIdx.x] = (r < ns && c < ns) ? A[(size_t)c * ld + r] : 0.0;
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    // A(c0 + x, r0 + k) = A(r0 + k, c0 + x) = a[x][k], strictly below the diagonal
    const int r = c0 + threadIdx.x, c = r0 + k;
    if (r < ns && c < r) A[(size_t)c * ld + r] = a[threadIdx.x][k];
  }
}

// cuSOLVER's multi-GPU library, opened on first use rather than linked: it
// needs a cuBLAS at least as new as the toolkit's, and a process that loaded
// an older cuBLAS first (a PyTorch wheel's) cannot load it.  Then only the
// eigensolves that need it fail, with the loader's message.
struct MgApi {
  decltype(&cusolverMgCreate) create = nullptr;
  decltype(&cusolverMgDestroy) destroy = nullptr;
  decltype(&cusolverMgDeviceSelect) device_select = nullptr;
  decltype(&cusolverMgCreateDeviceGrid) create_grid = nullptr;
  decltype(&cusolverMgDestroyGrid) destroy_grid = nullptr;
  decltype(&cusolverMgCreateMatrixDesc) create_desc = nullptr;
  decltype(&cusolverMgDestroyMatrixDesc) destroy_desc = nullptr;
  decltype(&cusolverMgSyevd_bufferSize) syevd_buffer = nullptr;
  decltype(&cusolverMgSyevd) syevd = nullptr;
  std::string error;
};
const MgApi& mg_api() {
  static const MgApi api = [] {
    MgApi a;
    void* lib = dlopen("libcusolverMg.so.11", RTLD_NOW | RTLD_LOCAL);
    if (!lib) {
      const char* e = dlerror();
      a.error = e ? e : "dlopen failed";
      return a;
    }
    auto get = [&](auto& f, const char* name) {
      f = reinterpret_cast<std::remove_reference_t<decltype(f)>>(dlsym(lib, name));
      if (!f && a.error.empty()) a.error = std::string("missing ") + name;
    };
    get(a.create, "cusolverMgCreate");
    get(a.destroy, "cusolverMgDestroy");
    get(a.device_select, "cusolverMgDeviceSelect");
    get(a.create_grid, "cusolverMgCreateDeviceGrid");
    get(a.destroy_grid, "cusolverMgDestroyGrid");
    get(a.create_desc, "cusolverMgCreateMatrixDesc");
    get(a.destroy_desc, "cusolverMgDestroyMatrixDesc");
    get(a.syevd_buffer, "cusolverMgSyevd_bufferSize");
    get(a.syevd, "cusolverMgSyevd");
    return a;
  }();
  return api;
}

// cuSOLVER multi-GPU objects of one eigensolve, released on every path
struct MgScratch {
  const MgApi& api;
  cusolverMgHandle_t h = nullptr;
  cudaLibMgGrid_t grid = nullptr;
  cudaLibMgMatrixDesc_t desc = nullptr;
  void* dwork = nullptr;
  explicit MgScratch(const MgApi& a) : api(a) {}
  ~MgScratch() {
    cudaFree(dwork);
    if (desc) api.destroy_desc(desc);
    if (grid) api.destroy_grid(grid);
    if (h) api.destroy(h);
  }
};

// cuSOLVER objects and buffers of one eigensolve, released on every path
struct EigScratch {
  cusolverDnHandle_t h = nullptr;
  cusolverDnParams_t prm = nullptr;
  void* dwork = nullptr;
  void* hwork = nullptr;
  int* dinfo = nullptr;
  ~EigScratch() {
    cudaFree(dwork);
    cudaFree(dinfo);
    std::free(hwork);
    if (prm) cusolverDnDestroyParams(prm);
    if (h) cusolverDnDestroy(h);
  }
};

}  // namespace

extern "C" int phx_smatrix_symmetrize(phx_smatrix* m) {
  PHX_ARG(nullptr, m, "phx_smatrix_symmetrize: null handle");
  phx_ctx* ctx = m->ctx;
  if (m->num_eig >= 0) {
    phx_set_error(ctx, PHX_ERR_STATE, "phx_smatrix_symmetrize: the matrix was diagonalized in place");
    return PHX_ERR_STATE;
  }
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  const int t = (m->ns + 31) / 32;
  symmetrize_kernel<<<dim3(t, t), dim3(32, 8), 0, ctx->stream>>>(m->ns, m->ns, m->d_A);
  PHX_CUDA(ctx, cudaGetLastError());
  PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PHX_OK;
}

int phx_smatrix_dot_launch(const phx_dot_args& a, cudaStream_t st, int* launches) {
  if (a.ncols <= 0 || a.ns <= 0 || a.nvec <= 0) return PHX_OK;
  if (launches) ++*launches;
  return a.nvec == 1 ? dot_launch<1>(a, st) : dot_launch<kDotVec>(a, st);
}

int phx_smatrix_diag_term_launch(int ns, int nT, int nvec, const double* lw, const double* x, double* y,
                                 const double* E, int finalize, cudaStream_t st) {
  const size_t n = (size_t)nvec * nT * 3 * ns;
  const int blocks = (int)std::min<size_t>(4096, (n + 255) / 256);
  diag_term_kernel<<<std::max(blocks, 1), 256, 0, st>>>(ns, nT, nvec, lw, x, y, E, finalize);
  return cudaGetLastError() == cudaSuccess ? PHX_OK : PHX_ERR_CUDA;
}

int phx_smatrix_set_diag_launch(int ns, long long ld, const double* diag, double* A, cudaStream_t st) {
  set_diag_kernel<<<(ns + 255) / 256, 256, 0, st>>>(ns, ld, diag, A);
  return cudaGetLastError() == cudaSuccess ? PHX_OK : PHX_ERR_CUDA;
}

extern "C" int phx_smatrix_num_states(const phx_smatrix* m) { return m ? m->ns : 0; }

extern "C" int phx_smatrix_diagonal(phx_smatrix* m, double* diag) {
  PHX_ARG(nullptr, m && diag, "phx_smatrix_diagonal: bad arguments");
  phx_ctx* ctx = m->ctx;
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  PHX_CUDA(ctx, cudaMemcpyAsync(diag, m->d_diag, sizeof(double) * m->ns, cudaMemcpyDeviceToHost, ctx->stream));
  PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PHX_OK;
}

extern "C" int phx_smatrix_get_rows(phx_smatrix* m, int row0, int nrows, double* out) {
  PHX_ARG(nullptr, m && out, "phx_smatrix_get_rows: bad arguments");
  phx_ctx* ctx = m->ctx;
  PHX_ARG(ctx, row0 >= 0 && nrows >= 0 && row0 + nrows <= m->ns, "phx_smatrix_get_rows: rows out of range");
  if (nrows == 0) return PHX_OK;
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t bytes = sizeof(double) * (size_t)nrows * m->ns;
  PHX_TRY(phx_ctx_reserve(ctx, &ctx->d_out, &ctx->out_bytes, bytes));
  double* d = static_cast<double*>(ctx->d_out);
  dim3 grid((m->ns + 31) / 32, (nrows + 31) / 32);
  rows_kernel<<<grid, dim3(32, 8), 0, ctx->stream>>>(m->ns, m->ns, m->d_A, row0, nrows, d);
  PHX_CUDA(ctx, cudaGetLastError());
  PHX_CUDA(ctx, cudaMemcpyAsync(out, d, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PHX_OK;
}

extern "C" int phx_smatrix_dot_d(phx_smatrix* m, int nvec, const double* x_d, int off_diagonal, double* y_d,
                                 float* ms) {
  PHX_ARG(nullptr, m && x_d && y_d && nvec >= 1, "phx_smatrix_dot: bad arguments");
  phx_ctx* ctx = m->ctx;
  if (m->num_eig >= 0 || m->omega) {
    phx_set_error(ctx, PHX_ERR_STATE,
                  m->num_eig >= 0 ? "phx_smatrix_dot: the matrix was diagonalized in place"
                                  : "phx_smatrix_dot: the matrix is scaled to Omega");
    return PHX_ERR_STATE;
  }
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (ms) {
    PHX_CUDA(ctx, cudaEventCreate(&e0));
    PHX_CUDA(ctx, cudaEventCreate(&e1));
    PHX_CUDA(ctx, cudaEventRecord(e0, st));
  }
  PHX_CUDA(ctx, cudaMemsetAsync(y_d, 0, sizeof(double) * nvec * 3 * (size_t)m->ns, st));
  phx_dot_args a{};
  a.ns = m->ns;
  a.ncols = m->ns;
  a.ld = m->ns;
  a.Sp = m->d_A;
  a.Sm = nullptr;
  a.tstride = 0;
  a.slab = 0;
  a.nb = m->nb;
  a.nT = 1;
  a.nvec = nvec;
  a.x = x_d;
  a.y = y_d;
  a.skip = off_diagonal ? 0 : 1;
  a.E = m->d_E;
  int rc = phx_smatrix_dot_launch(a, st, nullptr);
  if (rc != PHX_OK) {
    phx_set_error(ctx, rc, "phx_smatrix_dot: launch failed");
    return rc;
  }
  if (ms) {
    PHX_CUDA(ctx, cudaEventRecord(e1, st));
    PHX_CUDA(ctx, cudaEventSynchronize(e1));
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  return PHX_OK;
}

extern "C" int phx_smatrix_dot(phx_smatrix* m, int nvec, const double* x, int off_diagonal, double* y) {
  PHX_ARG(nullptr, m && x && y && nvec >= 1, "phx_smatrix_dot: bad arguments");
  phx_ctx* ctx = m->ctx;
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  const size_t n = (size_t)nvec * 3 * m->ns;
  if (m->xy_bytes < 2 * n * sizeof(double)) {
    cudaFree(m->d_xy);
    m->d_xy = nullptr;
    m->xy_bytes = 0;
    PHX_CUDA(ctx, cudaMalloc(&m->d_xy, 2 * n * sizeof(double)));
    m->xy_bytes = 2 * n * sizeof(double);
  }
  double* xd = m->d_xy;
  double* yd = m->d_xy + n;
  PHX_CUDA(ctx, cudaMemcpyAsync(xd, x, sizeof(double) * n, cudaMemcpyHostToDevice, ctx->stream));
  PHX_TRY(phx_smatrix_dot_d(m, nvec, xd, off_diagonal, yd, nullptr));
  PHX_CUDA(ctx, cudaMemcpyAsync(y, yd, sizeof(double) * n, cudaMemcpyDeviceToHost, ctx->stream));
  PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PHX_OK;
}

extern "C" int phx_smatrix_a2omega(phx_smatrix* m) {
  PHX_ARG(nullptr, m, "phx_smatrix_a2omega: null handle");
  phx_ctx* ctx = m->ctx;
  if (m->num_eig >= 0) {
    phx_set_error(ctx, PHX_ERR_STATE, "phx_smatrix_a2omega: the matrix was diagonalized in place");
    return PHX_ERR_STATE;
  }
  if (m->omega) return PHX_OK;   // already scaled, as the reference's isMatrixOmega
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const int ns = m->ns;
  double* term = nullptr;
  PHX_CUDA(ctx, phx_dev_alloc(ctx, (void**)&term, sizeof(double) * ns));
  poppm1_kernel<<<(ns + 255) / 256, 256, 0, st>>>(ns, m->d_E, m->temperature, term);
  a2omega_kernel<<<dim3((ns + 255) / 256, std::min(ns, 2048)), 256, 0, st>>>(ns, ns, term, m->d_A, m->d_diag);
  const cudaError_t e = cudaGetLastError();
  phx_dev_free(ctx, term);
  PHX_CUDA(ctx, e);
  PHX_CUDA(ctx, cudaStreamSynchronize(st));
  m->omega = 1;
  return PHX_OK;
}

// All eigenpairs through cuSOLVER's multi-GPU solver on a grid of this one
// device (the reference's distributed pdsyevd, scattering.cpp:816-910): its
// 64-bit workspace takes matrices that the single-GPU solvers refuse at their
// workspace query (48 000 states).  It reads the lower triangle, so the upper
// one (the reference's uplo = 'U') is first mirrored onto it.  Column blocks of
// a power of two up to 256 that divides ns (else one block): on one device the
// distributed matrix is then exactly the ns x ns column-major array.
// Eigenvalues ascending into w, eigenvectors over the matrix.
int eig_mg(phx_smatrix* m, std::vector<double>& w, int* info) {
  phx_ctx* ctx = m->ctx;
  const int ns = m->ns;
  cudaStream_t st = ctx->stream;
  if (!mg_api().error.empty()) {
    phx_set_error(ctx, PHX_ERR_CUDA, "phx_smatrix_diagonalize: cuSOLVER's multi-GPU solver, needed for " +
                                         std::to_string(ns) + " states, could not be loaded: " + mg_api().error);
    return PHX_ERR_CUDA;
  }
  const int t = (ns + 31) / 32;
  mirror_upper_kernel<<<dim3(t, t), dim3(32, 8), 0, st>>>(ns, ns, m->d_A);
  PHX_CUDA(ctx, cudaGetLastError());
  PHX_CUDA(ctx, cudaStreamSynchronize(st));
  auto mg = [&](cusolverStatus_t s, const char* what) {
    if (s == CUSOLVER_STATUS_SUCCESS) return PHX_OK;
    phx_set_error(ctx, PHX_ERR_CUDA, std::string("phx_smatrix_diagonalize: ") + what + " failed (cusolver status " +
                                         std::to_string((int)s) + ")");
    return PHX_ERR_CUDA;
  };
  int cb = ns;
  for (int b = 256; b >= 32; b /= 2)
    if (ns % b == 0) {
      cb = b;
      break;
    }
  const MgApi& api = mg_api();
  MgScratch z(api);
  int dev = ctx->device;
  PHX_TRY(mg(api.create(&z.h), "cusolverMgCreate"));
  PHX_TRY(mg(api.device_select(z.h, 1, &dev), "cusolverMgDeviceSelect"));
  PHX_TRY(mg(api.create_grid(&z.grid, 1, 1, &dev, CUDALIBMG_GRID_MAPPING_COL_MAJOR), "cusolverMgCreateDeviceGrid"));
  PHX_TRY(mg(api.create_desc(&z.desc, ns, ns, ns, cb, CUDA_R_64F, z.grid), "cusolverMgCreateMatrixDesc"));
  void* arrA[1] = {m->d_A};
  w.assign(ns, 0.0);
  int64_t lwork = 0;
  PHX_TRY(mg(api.syevd_buffer(z.h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, ns, arrA, 1, 1, z.desc, w.data(),
                              CUDA_R_64F, CUDA_R_64F, &lwork),
             "cusolverMgSyevd_bufferSize"));
  PHX_CUDA(ctx, cudaMalloc(&z.dwork, sizeof(double) * (size_t)std::max<int64_t>(lwork, 1)));
  void* arrW[1] = {z.dwork};
  PHX_TRY(mg(api.syevd(z.h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, ns, arrA, 1, 1, z.desc, w.data(),
                       CUDA_R_64F, CUDA_R_64F, arrW, lwork, info),
             "cusolverMgSyevd"));
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  PHX_CUDA(ctx, cudaDeviceSynchronize());
  return PHX_OK;
}

extern "C" int phx_smatrix_diagonalize(phx_smatrix* m, int num_eigenvalues, double* eigenvalues, int* num_found) {
  PHX_ARG(nullptr, m && eigenvalues && num_found, "phx_smatrix_diagonalize: bad arguments");
  phx_ctx* ctx = m->ctx;
  const int ns = m->ns;
  PHX_ARG(ctx, num_eigenvalues <= ns,
          "You have requested to calculate more relaxons eigenvalues than your number of particle states.");
  if (m->num_eig >= 0) {
    phx_set_error(ctx, PHX_ERR_STATE, "phx_smatrix_diagonalize: the matrix was diagonalized already");
    return PHX_ERR_STATE;
  }
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  if (!m->d_W) PHX_CUDA(ctx, cudaMalloc(&m->d_W, sizeof(double) * ns));
  PHX_CUDA(ctx, cudaMemsetAsync(m->d_W, 0, sizeof(double) * ns, st));
  EigScratch z;
  auto solver = [&](cusolverStatus_t s, const char* what) {
    if (s == CUSOLVER_STATUS_SUCCESS) return PHX_OK;
    phx_set_error(ctx, PHX_ERR_CUDA, std::string("phx_smatrix_diagonalize: ") + what + " failed (cusolver status " +
                                         std::to_string((int)s) + ")");
    return PHX_ERR_CUDA;
  };
  PHX_TRY(solver(cusolverDnCreate(&z.h), "cusolverDnCreate"));
  PHX_TRY(solver(cusolverDnSetStream(z.h, st), "cusolverDnSetStream"));
  PHX_TRY(solver(cusolverDnCreateParams(&z.prm), "cusolverDnCreateParams"));
  // the upper triangle, as the reference's pdsyevd / pdsyevr with uplo = 'U'
  const cublasFillMode_t uplo = CUBLAS_FILL_MODE_UPPER;
  const cusolverEigMode_t jobz = CUSOLVER_EIG_MODE_VECTOR;
  const bool some = num_eigenvalues > 0 && num_eigenvalues != ns;
  double vl = -1.0, vu = 0.0;
  int64_t meig = ns;
  size_t dws = 0, hws = 0;
  const char* force_mg = std::getenv("PHX_EIG_MG");
  cusolverStatus_t qs = CUSOLVER_STATUS_INVALID_VALUE;
  if (!(force_mg && force_mg[0] == '1')) {
    if (some)
      qs = cusolverDnXsyevdx_bufferSize(z.h, z.prm, jobz, CUSOLVER_EIG_RANGE_I, uplo, ns, CUDA_R_64F, m->d_A, ns, &vl,
                                        &vu, 1, num_eigenvalues, &meig, CUDA_R_64F, m->d_W, CUDA_R_64F, &dws, &hws);
    else
      qs = cusolverDnXsyevd_bufferSize(z.h, z.prm, jobz, uplo, ns, CUDA_R_64F, m->d_A, ns, CUDA_R_64F, m->d_W,
                                       CUDA_R_64F, &dws, &hws);
  }
  if (qs == CUSOLVER_STATUS_INVALID_VALUE) {
    // refused at the workspace query (or PHX_EIG_MG=1): all eigenpairs by the
    // multi-GPU solver on this device, the smallest num_eigenvalues kept
    std::vector<double> w;
    int info = 0;
    const int rc = eig_mg(m, w, &info);
    m->num_eig = 0;   // the matrix is overwritten from here on, whatever the outcome
    if (rc != PHX_OK) return rc;
    if (info != 0) {
      phx_set_error(ctx, info > 0 ? PHX_ERR_NOCONV : PHX_ERR_ARG,
                    "phx_smatrix_diagonalize: eigensolver info = " + std::to_string(info));
      return info > 0 ? PHX_ERR_NOCONV : PHX_ERR_ARG;
    }
    const int k = some ? num_eigenvalues : ns;
    PHX_CUDA(ctx, cudaMemcpy(m->d_W, w.data(), sizeof(double) * ns, cudaMemcpyHostToDevice));
    std::memcpy(eigenvalues, w.data(), sizeof(double) * k);
    m->num_eig = k;
    *num_found = k;
    return PHX_OK;
  }
  PHX_TRY(solver(qs, some ? "cusolverDnXsyevdx_bufferSize" : "cusolverDnXsyevd_bufferSize"));
  PHX_CUDA(ctx, cudaMalloc(&z.dwork, std::max<size_t>(dws, 8)));
  PHX_CUDA(ctx, cudaMalloc(&z.dinfo, sizeof(int)));
  z.hwork = std::malloc(std::max<size_t>(hws, 8));
  PHX_ARG(ctx, z.hwork, "phx_smatrix_diagonalize: host workspace allocation failed");
  if (some)
    PHX_TRY(solver(cusolverDnXsyevdx(z.h, z.prm, jobz, CUSOLVER_EIG_RANGE_I, uplo, ns, CUDA_R_64F, m->d_A, ns, &vl, &vu,
                                     1, num_eigenvalues, &meig, CUDA_R_64F, m->d_W, CUDA_R_64F, z.dwork, dws, z.hwork,
                                     hws, z.dinfo),
                   "cusolverDnXsyevdx"));
  else
    PHX_TRY(solver(cusolverDnXsyevd(z.h, z.prm, jobz, uplo, ns, CUDA_R_64F, m->d_A, ns, CUDA_R_64F, m->d_W,
                                    CUDA_R_64F, z.dwork, dws, z.hwork, hws, z.dinfo),
                   "cusolverDnXsyevd"));
  int info = 0;
  PHX_CUDA(ctx, cudaMemcpyAsync(&info, z.dinfo, sizeof(int), cudaMemcpyDeviceToHost, st));
  PHX_CUDA(ctx, cudaStreamSynchronize(st));
  // the matrix is overwritten from here on, whatever the outcome
  m->num_eig = 0;
  if (info != 0) {
    phx_set_error(ctx, info > 0 ? PHX_ERR_NOCONV : PHX_ERR_ARG,
                  "phx_smatrix_diagonalize: eigensolver info = " + std::to_string(info));
    return info > 0 ? PHX_ERR_NOCONV : PHX_ERR_ARG;
  }
  m->num_eig = (int)meig;
  PHX_CUDA(ctx, cudaMemcpyAsync(eigenvalues, m->d_W, sizeof(double) * meig, cudaMemcpyDeviceToHost, st));
  PHX_CUDA(ctx, cudaStreamSynchronize(st));
  *num_found = (int)meig;
  return PHX_OK;
}

extern "C" int phx_smatrix_relaxon_solve(phx_smatrix* m, int nvec, const double* x, double* y) {
  PHX_ARG(nullptr, m && x && y && nvec >= 1, "phx_smatrix_relaxon_solve: bad arguments");
  phx_ctx* ctx = m->ctx;
  if (m->num_eig < 0) {
    phx_set_error(ctx, PHX_ERR_STATE, "phx_smatrix_relaxon_solve called before phx_smatrix_diagonalize");
    return PHX_ERR_STATE;
  }
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = ctx->stream;
  const int ns = m->ns;
  const size_t n = (size_t)nvec * 3 * ns;
  double* d = nullptr;   // x, the relaxon populations, y
  PHX_CUDA(ctx, phx_dev_alloc(ctx, (void**)&d, 3 * n * sizeof(double)));
  double *xd = d, *rd = d + n, *yd = d + 2 * n;
  cudaError_t e = cudaMemcpyAsync(xd, x, sizeof(double) * n, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(rd, 0, 2 * n * sizeof(double), st);
  int rc = PHX_OK;
  if (e == cudaSuccess && m->num_eig > 0) {
    relaxon_project_kernel<<<m->num_eig, 256, 0, st>>>(ns, ns, m->d_A, m->d_W, nvec, xd, rd);
    e = cudaGetLastError();
    if (e == cudaSuccess) {
      // back to the states: y = Theta r over the computed eigenvectors (:350-380)
      phx_dot_args a{};
      a.ns = ns;
      a.ncols = m->num_eig;
      a.ld = ns;
      a.Sp = m->d_A;
      a.nb = m->nb;
      a.nT = 1;
      a.nvec = nvec;
      a.x = rd;
      a.y = yd;
      a.skip = 2;
      a.E = m->d_E;
      rc = phx_smatrix_dot_launch(a, st, nullptr);
    }
  }
  if (e == cudaSuccess && rc == PHX_OK) e = cudaMemcpyAsync(y, yd, sizeof(double) * n, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  phx_dev_free(ctx, d);
  PHX_CUDA(ctx, e);
  if (rc != PHX_OK) phx_set_error(ctx, rc, "phx_smatrix_relaxon_solve: launch failed");
  return rc;
}

extern "C" int phx_smatrix_destroy(phx_smatrix* m) {
  if (!m) return PHX_OK;
  if (m->ctx) cudaSetDevice(m->ctx->device);
  cudaFree(m->d_W);
  cudaFree(m->d_A);
  cudaFree(m->d_E);
  cudaFree(m->d_diag);
  cudaFree(m->d_xy);
  delete m;
  return PHX_OK;
}
