// Internal definitions shared by the translation units of libphx.
#pragma once
#include <cuda_runtime.h>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/phx_abi.h"

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
void phx_set_error(const phx_ctx* ctx, int code, const std::string& msg);

#define PHX_CUDA(ctx, call)                                                          \
  do {                                                                               \
    cudaError_t _e = (call);                                                         \
    if (_e != cudaSuccess) {                                                         \
      phx_set_error((ctx), PHX_ERR_CUDA,                                             \
                    std::string(#call) + ": " + cudaGetErrorString(_e) + " at " +    \
                        __FILE__ + ":" + std::to_string(__LINE__));                  \
      return PHX_ERR_CUDA;                                                           \
    }                                                                                \
  } while (0)

#define PHX_ARG(ctx, cond, msg)                       \
  do {                                                \
    if (!(cond)) {                                    \
      phx_set_error((ctx), PHX_ERR_ARG, (msg));       \
      return PHX_ERR_ARG;                             \
    }                                                 \
  } while (0)

#define PHX_TRY(x)             \
  do {                         \
    int _rc = (x);             \
    if (_rc != PHX_OK) return _rc; \
  } while (0)

// ---------------------------------------------------------------------------
// handles
// ---------------------------------------------------------------------------
struct phx_ctx {
  int device = 0;
  int num_sms = 148;
  cudaStream_t stream = nullptr;
  mutable std::string last_error;
  mutable int last_status = 0;
  // device status word written by kernels (non-convergence, mesh misses)
  int* d_status = nullptr;
  // builder scratch and output staging, kept for the context's lifetime so
  // that objects created and destroyed between calls reuse them (calls on one
  // context run on its one stream, in order)
  void* d_scratch = nullptr;
  size_t scratch_bytes = 0;
  void* d_out = nullptr;
  size_t out_bytes = 0;
};

// grow-only device buffers of a context
int phx_ctx_reserve(phx_ctx* ctx, void** buf, size_t* have, size_t bytes);

// Device memory of the objects (band structures, couplings, Hamiltonians):
// stream-ordered allocations on the context's stream from the device's default
// memory pool, whose release threshold phx_ctx_create raises so that freed
// blocks stay in the pool.  Objects created and destroyed between calls then
// neither map memory nor synchronise the device.
cudaError_t phx_dev_alloc(phx_ctx* ctx, void** p, size_t bytes);
void phx_dev_free(phx_ctx* ctx, void* p);

// Records e on st; while st is being captured into a graph the record becomes
// an external event node, so that the event times the graph's replays.
inline cudaError_t phx_record_event(cudaEvent_t e, cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaStreamIsCapturing(st, &cs);
  return cs == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(e, st, cudaEventRecordExternal)
                                             : cudaEventRecord(e, st);
}

struct phx_ph_h0 {
  phx_ctx* ctx = nullptr;
  int nat = 0, nb = 0, numR = 0;
  double cell[9];             // lattice vectors as columns
  double recip[9];            // reciprocal vectors as columns
  std::vector<double> masses; // per band
  double* d_R = nullptr;      // (numR,3) Wigner-Seitz vectors grouped by atom pair
  int* d_pofs = nullptr;      // (nat*nat+1) offsets of each atom pair's R range
  double* d_wblk = nullptr;   // (numR,9) weight * 3x3 force-constant block
  double* d_masses = nullptr; // (nb)
};

struct phx_bands {
  phx_ctx* ctx = nullptr;
  int nb = 0, nq = 0;
  int mesh[3] = {0, 0, 0};
  double recip[9];            // reciprocal cell, columns = b vectors
  double* d_E = nullptr;      // (nq,nb)
  double* d_U = nullptr;      // (nq,nb,nb) complex, mass-scaled
  double* d_vg = nullptr;     // (nq,nb,3) or null
  double* d_q = nullptr;      // (nq,3) Cartesian mesh points
  float* d_U32 = nullptr;     // (nq,nb,nb) complex fp32 copy for the split path
  int* d_q1_order = nullptr;  // (nq) q1 visiting order of the split path
  double emax = -1.0;         // largest |E| of the mesh (split path), < 0 until computed
};

// CUDA graphs of the builder, owned by the v3 object (builder.cu)
struct phx_builder_graphs;
void phx_builder_release(phx_v3* v);

struct phx_v3 {
  phx_ctx* ctx = nullptr;
  int nat = 0, nb = 0, nr2 = 0, nr3 = 0;
  int precision = PHX_PREC_FP64;
  std::vector<double> R2, R3;
  double* d_D3w = nullptr;     // (nr3,nr2,nb,nb,nb) weights folded (w2*w3*w3)
  double* d_D3raw = nullptr;   // (nb,nb,nb,nr3,nr2) for the cacheD3 API path
  double* d_w2 = nullptr;      // (nr2,nat,nat)
  double* d_w3 = nullptr;      // (nr3,nat,nat)
  double* d_R2 = nullptr;      // (nr2,3)
  double* d_R3 = nullptr;      // (nr3,3)
  double* d_plus = nullptr;    // cached D3+ (nb,nb,nb,nr3) complex
  double* d_mins = nullptr;    // cached D3- (nb,nb,nb,nr3) complex
  bool cached = false;
  double q2_cached[3];
  phx_builder_graphs* graphs = nullptr;
  // non-zero (r3, r2) blocks of d_D3w (many-branch builder): for r3, the r2 in
  // d_r2_list[d_r2_ofs[r3] .. d_r2_ofs[r3+1]); built on first use
  int* d_r2_ofs = nullptr;
  int* d_r2_list = nullptr;
  int r2_max_list = 0;
};

int phx_scratch_reserve(phx_v3* v3, size_t bytes);

// screening network (mlp.cu): forward pass of device inputs, on the context's stream
int phx_mlp_forward_device(phx_mlp* net, long long B, const float* dX, float* dY);
int phx_mlp_num_inputs(const phx_mlp* net);
phx_ctx* phx_mlp_context(const phx_mlp* net);

// Cartesian coordinates (n,3) of a Gamma-centred mesh (recip: columns = b vectors)
void phx_mesh_cartesian(const int* mesh, const double* recip, std::vector<double>& q);

struct phx_el_h0 {
  phx_ctx* ctx = nullptr;
  int nw = 0, nR = 0;
  double cell[9];             // lattice vectors as columns
  double recip[9];            // reciprocal vectors as columns
  double* d_R = nullptr;      // (nR,3) Bravais vectors (Bohr)
  double* d_deg = nullptr;    // (nR) degeneracies
  double* d_H = nullptr;      // (nR,nw,nw) complex Wannier Hamiltonian (Ry)
};

struct phx_elph {
  phx_ctx* ctx = nullptr;
  int nw = 0, nph = 0, nRe = 0, nRp = 0;
  double* d_Re = nullptr;     // (nRe,3)
  double* d_degE = nullptr;   // (nRe)
  double* d_Rp = nullptr;     // (nRp,3)
  double* d_degP = nullptr;   // (nRp)
  float* d_g = nullptr;       // (nRe,nRp,nph,nw,nw) complex FP32 coupling in the Wannier basis
  double* d_cached = nullptr; // (nRp,nph,nw,nw) complex: cacheElPh of the last k1 (b1 < nb1)
  int nb1 = 0;                // bands of the cached k1
  int precision = PHX_PREC_FP64;  // of the Re and Rp transforms in phx_el_linewidths
  uint8_t* d_gimg = nullptr;  // split path: BF16 hi/lo tile image of g (built on first use)
  uint8_t* d_kimg = nullptr;  // split path: phase image of a k1 batch
  void* d_scratch = nullptr;  // builder scratch (grown on demand)
  size_t scratch_bytes = 0;
};

// ---------------------------------------------------------------------------
// scattering matrix (smatrix.cu): column-major blocks, element (row, col) at
// col * ld + row, with row and col the state index iq * nb + ib.
// ---------------------------------------------------------------------------
struct phx_smatrix {
  phx_ctx* ctx = nullptr;
  int nq = 0, nb = 0, ns = 0;
  int mesh[3] = {0, 0, 0};
  double* d_A = nullptr;      // (ns, ns) column-major
  double* d_E = nullptr;      // (ns) energies (exclusions of the dot product)
  double* d_diag = nullptr;   // (ns) the diagonal: linewidths x n(n+1), not averaged
  double* d_xy = nullptr;     // staging of x and y for phx_smatrix_dot
  size_t xy_bytes = 0;
  double temperature = 0.0;   // Ry, the matrix's one temperature
  int omega = 0;              // 1: scaled to Omega (phx_smatrix_a2omega)
  int num_eig = -1;           // >= 0: d_A holds that many eigenvectors (phx_smatrix_diagonalize)
  double* d_W = nullptr;      // (ns) eigenvalues, ascending
};

// y += (block of a scattering matrix) x, for x and y (nvec, nT, 3, ns) on the device.
struct phx_dot_args {
  int ns;                  // rows (states)
  int ncols;               // columns of the block
  long long ld;
  const double* Sp;        // the block; temperature c at Sp + c * tstride
  const double* Sm;        // slab of "-" rates, or null
  size_t tstride;
  // slab = 1: column k = j nb + b2 is the state (q2_first + j) nb + b2 in Sp
  // and (-(q2_first + j)) nb + b2 in Sm; slab = 0: column k is the state k
  int slab, q2_first, nb, n0, n1, n2;
  int nT, nvec;
  const double* x;
  double* y;
  // skip = 0: the element whose column state is the row state is left out
  // (the off-diagonal part); 1: rows and columns of excluded states are left
  // out (ScatteringMatrix::dot of a stored matrix); 2: nothing left out
  int skip;
  const double* E;         // (ns), for skip = 1
};
int phx_smatrix_dot_launch(const phx_dot_args& a, cudaStream_t st, int* launches);
// Matrix output of the split pair kernel, in the layouts of the FP64 matrix
// modes: full = 1, `plus` is the whole matrix (one temperature); full = 0,
// `plus` and `minus` are the two slabs of the chunk, columns j nb + b2 with
// j = q2 - q2_first, temperature t at t * tstride.
struct phx_split_matrix {
  double* plus;
  double* minus;
  long long ld;
  size_t tstride;
  int full;
};
// y (nvec, nT, 3, ns) += lw (nT, ns) * x; then, with finalize, y = 0 on excluded states
int phx_smatrix_diag_term_launch(int ns, int nT, int nvec, const double* lw, const double* x, double* y,
                                 const double* E, int finalize, cudaStream_t st);
// A(s, s) = diag(s)
int phx_smatrix_set_diag_launch(int ns, long long ld, const double* diag, double* A, cudaStream_t st);

// kernels implemented in harmonic.cu, used by the ABI layer
int phx_launch_ph_bands(phx_ph_h0* h0, int nq, const double* d_q, double* d_E, double* d_U,
                        double* d_vg, int mass_scaling);
