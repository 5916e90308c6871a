// Context, error reporting, and host-side harmonic setup of libphx.
//
// phx_ws_reorder restates PhononH0::setAcousticSumRule "simple"
// (src/harmonic/phonon_h0_sum_rule.cpp:45-79), wsInit/wsWeight
// (src/harmonic/phonon_h0.cpp:426-535) and reorderDynamicalMatrix
// (src/harmonic/phonon_h0.cpp:672-771): the same weights, the same ordering of
// the (R, atom pair) list, so mat2R can be compared element by element.
#include <cmath>
#include <cstring>
#include <mutex>

#include "phx_internal.h"

namespace {
std::mutex g_err_mutex;
std::string g_last_error;
int g_last_status = 0;
}  // namespace

void phx_set_error(const phx_ctx* ctx, int code, const std::string& msg) {
  if (ctx) {
    ctx->last_error = msg;
    ctx->last_status = code;
  }
  std::lock_guard<std::mutex> lk(g_err_mutex);
  g_last_error = msg;
  g_last_status = code;
}

extern "C" const char* phx_version(void) { return "phx 0.1 (sm_100a)"; }

extern "C" int phx_last_error(const phx_ctx* ctx, char* buf, size_t len) {
  std::string msg;
  int st;
  if (ctx) {
    msg = ctx->last_error;
    st = ctx->last_status;
  } else {
    std::lock_guard<std::mutex> lk(g_err_mutex);
    msg = g_last_error;
    st = g_last_status;
  }
  if (buf && len) {
    std::strncpy(buf, msg.c_str(), len - 1);
    buf[len - 1] = 0;
  }
  return st;
}

extern "C" int phx_ctx_create(int device, phx_ctx** out) {
  PHX_ARG(nullptr, out != nullptr, "phx_ctx_create: out is NULL");
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    phx_set_error(nullptr, PHX_ERR_NODEV,
                  std::string("no CUDA device: ") + cudaGetErrorString(e));
    return PHX_ERR_NODEV;
  }
  PHX_ARG(nullptr, device >= 0 && device < n, "phx_ctx_create: bad device index");
  PHX_CUDA(nullptr, cudaSetDevice(device));
  cudaDeviceProp prop;
  PHX_CUDA(nullptr, cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) {
    phx_set_error(nullptr, PHX_ERR_NODEV, "libphx is built for sm_100a; device is sm_" +
                                              std::to_string(prop.major * 10 + prop.minor));
    return PHX_ERR_NODEV;
  }
  phx_ctx* c = new phx_ctx;
  c->device = device;
  c->num_sms = prop.multiProcessorCount;
  cudaError_t e2 = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (e2 == cudaSuccess) {
    // keep freed object memory in this process's pool (phx_dev_alloc)
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t keep = ~uint64_t(0);
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
  }
  if (e2 == cudaSuccess) e2 = cudaMalloc(&c->d_status, 64 * sizeof(int));
  if (e2 == cudaSuccess) e2 = cudaMemset(c->d_status, 0, 64 * sizeof(int));
  if (e2 != cudaSuccess) {
    phx_set_error(nullptr, PHX_ERR_CUDA, cudaGetErrorString(e2));
    delete c;
    return PHX_ERR_CUDA;
  }
  *out = c;
  return PHX_OK;
}

extern "C" int phx_ctx_destroy(phx_ctx* ctx) {
  if (!ctx) return PHX_OK;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->d_status) cudaFree(ctx->d_status);
  cudaFree(ctx->d_scratch);
  cudaFree(ctx->d_out);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  // The struct itself stays allocated (a few hundred bytes): objects that
  // outlive their context free their memory through it, on the default stream.
  ctx->stream = nullptr;
  ctx->d_status = nullptr;
  ctx->d_scratch = ctx->d_out = nullptr;
  ctx->scratch_bytes = ctx->out_bytes = 0;
  return PHX_OK;
}

extern "C" int phx_ctx_synchronize(phx_ctx* ctx) {
  PHX_ARG(nullptr, ctx, "null context");
  PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return PHX_OK;
}

// ---------------------------------------------------------------------------
// Wigner-Seitz reordering (host, FP64)
// ---------------------------------------------------------------------------
namespace {
double ws_weight(const double r[3], const std::vector<double>& rws) {
  int nreq = 1;
  const size_t n = rws.size() / 3;
  for (size_t i = 0; i < n; ++i) {
    const double* g = &rws[3 * i];
    const double ck = (r[0] * g[0] + r[1] * g[1] + r[2] * g[2]) -
                      (g[0] * g[0] + g[1] * g[1] + g[2] * g[2]) / 2.0;
    if (ck > 1.0e-5) return 0.0;
    if (std::fabs(ck) <= 1.0e-5) ++nreq;
  }
  return 1.0 / double(nreq);
}
}  // namespace

extern "C" int phx_ws_reorder(int nat, const double* cell, const double* pos, const int* grid,
                              const double* fc_in, int* numR, double* R, double* w,
                              double* mat2R) {
  PHX_ARG(nullptr, nat > 0 && cell && pos && grid && fc_in && numR, "phx_ws_reorder: bad args");
  const int g1 = grid[0], g2 = grid[1], g3 = grid[2];
  PHX_ARG(nullptr, g1 > 0 && g2 > 0 && g3 > 0, "phx_ws_reorder: bad grid");
  const int nb = 3 * nat;
  const size_t nfc = (size_t)9 * g1 * g2 * g3 * nat * nat;
  std::vector<double> fc(fc_in, fc_in + nfc);
  auto FI = [&](int i, int j, int m1, int m2, int m3, int a, int b) {
    return ((((((size_t)i * 3 + j) * g1 + m1) * g2 + m2) * g3 + m3) * nat + a) * nat + b;
  };
  // simple acoustic sum rule on the force constants
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j)
      for (int a = 0; a < nat; ++a) {
        double s = 0.0;
        for (int b = 0; b < nat; ++b)
          for (int m1 = 0; m1 < g1; ++m1)
            for (int m2 = 0; m2 < g2; ++m2)
              for (int m3 = 0; m3 < g3; ++m3) s += fc[FI(i, j, m1, m2, m3, a, b)];
        fc[FI(i, j, 0, 0, 0, a, a)] -= s;
      }
  // Wigner-Seitz neighbours of the supercell lattice
  std::vector<double> rws;
  for (int i1 = -2; i1 <= 2; ++i1)
    for (int i2 = -2; i2 <= 2; ++i2)
      for (int i3 = -2; i3 <= 2; ++i3) {
        double t[3];
        for (int c = 0; c < 3; ++c)
          t[c] = cell[c * 3 + 0] * g1 * i1 + cell[c * 3 + 1] * g2 * i2 + cell[c * 3 + 2] * g3 * i3;
        if (t[0] * t[0] + t[1] * t[1] + t[2] * t[2] > 1.0e-6) rws.insert(rws.end(), t, t + 3);
      }
  const int B1 = 2 * g1, B2 = 2 * g2, B3 = 2 * g3;
  const int S1 = 2 * B1 + 1, S2 = 2 * B2 + 1, S3 = 2 * B3 + 1;
  std::vector<double> wc((size_t)S1 * S2 * S3 * nat * nat);
  auto WI = [&](int n1, int n2, int n3, int a, int b) {
    return ((((size_t)(n3 + B3) * S2 + (n2 + B2)) * S1 + (n1 + B1)) * nat + b) * nat + a;
  };
  for (int a = 0; a < nat; ++a)
    for (int b = 0; b < nat; ++b) {
      double total = 0.0;
      for (int n1 = -B1; n1 <= B1; ++n1)
        for (int n2 = -B2; n2 <= B2; ++n2)
          for (int n3 = -B3; n3 <= B3; ++n3) {
            double r[3];
            for (int c = 0; c < 3; ++c)
              r[c] = n1 * cell[c * 3 + 0] + n2 * cell[c * 3 + 1] + n3 * cell[c * 3 + 2] +
                     pos[a * 3 + c] - pos[b * 3 + c];
            const double x = ws_weight(r, rws);
            wc[WI(n1, n2, n3, a, b)] = x;
            total += x;
          }
      if (std::fabs(total - (double)g1 * g2 * g3) > 1.0e-8) {
        phx_set_error(nullptr, PHX_ERR_ARG, "phx_ws_reorder: Wigner-Seitz weights do not sum to the grid size");
        return PHX_ERR_ARG;
      }
    }
  int iR = 0;
  for (int n3 = -B3; n3 <= B3; ++n3)
    for (int n2 = -B2; n2 <= B2; ++n2)
      for (int n1 = -B1; n1 <= B1; ++n1)
        for (int b = 0; b < nat; ++b)
          for (int a = 0; a < nat; ++a) {
            const double wt = wc[WI(n1, n2, n3, a, b)];
            if (wt <= 0.0) continue;
            if (R && w && mat2R) {
              w[iR] = wt;
              for (int c = 0; c < 3; ++c)
                R[iR * 3 + c] = n1 * cell[c * 3 + 0] + n2 * cell[c * 3 + 1] + n3 * cell[c * 3 + 2];
              double* M = mat2R + (size_t)iR * nb * nb;
              std::memset(M, 0, sizeof(double) * nb * nb);
              const int m1 = ((n1 % g1) + g1) % g1, m2 = ((n2 % g2) + g2) % g2,
                        m3 = ((n3 % g3) + g3) % g3;
              for (int j = 0; j < 3; ++j)
                for (int i = 0; i < 3; ++i)
                  M[(3 * a + i) * nb + 3 * b + j] += fc[FI(i, j, m1, m2, m3, a, b)];
            }
            ++iR;
          }
  *numR = iR;
  return PHX_OK;
}

cudaError_t phx_dev_alloc(phx_ctx* ctx, void** p, size_t bytes) {
  return cudaMallocAsync(p, bytes > 0 ? bytes : 1, ctx->stream);
}

void phx_dev_free(phx_ctx* ctx, void* p) {
  if (!p) return;
  if (ctx->stream) cudaFreeAsync(p, ctx->stream);
  else cudaFree(p);
}

int phx_ctx_reserve(phx_ctx* ctx, void** buf, size_t* have, size_t bytes) {
  if (*have >= bytes && *buf) return PHX_OK;
  PHX_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  cudaFree(*buf);
  *buf = nullptr;
  *have = 0;
  PHX_CUDA(ctx, cudaMalloc(buf, bytes));
  *have = bytes;
  return PHX_OK;
}
