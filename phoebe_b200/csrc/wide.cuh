// Builder for cells with many branches (wide.cu): arguments and launchers,
// shared with the host orchestration in builder.cu.
#pragma once
#include <cstdint>

#include "pair_common.cuh"

namespace wide {

constexpr int kMaxNb = 48;      // branches (16 atoms)
constexpr int kQ1 = 8;          // q1 per work item of the split kernel (its N = 16 MMA columns)

struct Args {
  pairc::MeshArgs m;
  int nr3;
  const double* R3;
  const double2* Dp;          // [j][r3][a][b2][c] FP64, j = q2 - q2_first
  int q2_first, q2_count;
  const int* q1_order;        // (nq) q1 order: tile t = q1_order[t*nq1 ...]
  int nq1;                    // q1 per work item
  int ntiles;
  const double* win_energy;   // (nq) or null: pair (q1, q2) iff energy[q2] <= cut[q1]
  const double* win_cut;
  double* lw;                 // (nq, nb, nT) partial linewidths (FP64 atomics)
  unsigned* counter;          // work queue, zero at launch
  int* status;
  // screening: skip[(q2 - skip_base) * nq + q1] != 0 drops the vertex (q1, q2), or null
  const uint8_t* skip;
  int skip_base;
  // split path
  const uint8_t* img;         // A-operand tiles [j][b2][mt][kc], hi then lo
  const float2* U32;          // (nq, nb, nb) FP32 eigenvectors
  int Kp, mtiles, fp16;
  const unsigned* dmax;
  int rt, qp;                 // split kernel tile shape: register tile (2 or 4), q1 planes per contraction pass
};

// FP64 kernel: q1 per item for this nb and nr3 (0: too large), and its shared memory
int fp64_q1(int nb, int nr3);
size_t fp64_smem(int nq1, int nb, int nr3);
// split kernel: shared memory for qp q1 planes per contraction pass (0 if it
// does not fit), the default tile shape, and the bytes of one q2 of the image
size_t split_smem(int nb, int Kp, int qp);
int split_default_qp(int nb, int Kp);
size_t split_img_bytes(int nb, int Kp);
int split_kp(int nr3);
int split_mtiles(int nb);

// persistent pair kernel over the items (q2 of the chunk) x (q1 tiles); grid = CTAs
cudaError_t launch_fp64(const Args& A, int grid, cudaStream_t st);
cudaError_t launch_split(const Args& A, int grid, cudaStream_t st);
cudaError_t set_attributes(int nb, int nr3, bool split);   // for every tile shape
int blocks_per_sm(int nb, int nr3, bool split);
// R2 fold of a chunk of q2 (sparse over the non-zero (r3, r2) blocks)
size_t fold_smem(int nb, int max_list);
cudaError_t launch_fold(int nb, int nr2, int nr3, const double* D3w, const int* r2_ofs, const int* r2_list,
                        int max_list, const double* R2, const double* R3, const double* qcart, const double2* U,
                        int q2_first, int q2_count, double2* Dp, unsigned* dmax, cudaStream_t st);
// FP64 Dp of a chunk -> split A-operand tiles (FP16 or BF16 hi/lo)
cudaError_t launch_convert(int nb, int nr3, int Kp, int q2_count, const double2* Dp, uint8_t* img, int fp16,
                           const unsigned* dmax, cudaStream_t st);
// U32 = (float2) U, n complex entries
cudaError_t launch_u32(const double2* U, float2* U32, size_t n, cudaStream_t st);
// screening: features X ((q2 - q2_first) * nq + q1, 12) of the (q1, q2) pairs of a q2 range
constexpr int kPairFeatures = 12;
cudaError_t launch_pair_features(int nq, int nb, int n0, int n1, int n2, const double* E, double emax, int q2_first,
                                 int q2_count, float* X, cudaStream_t st);
// skip[i] = y[i] < log10_threshold
cudaError_t launch_screen_mask(size_t n, const float* y, float log10_threshold, uint8_t* skip,
                               unsigned long long* nskip, cudaStream_t st);
// flags[r3 * nr2 + r2] = 1 for the non-zero blocks of D3w (nr3, nr2, nb^3)
cudaError_t launch_nonzero_blocks(int nb, int nr3, int nr2, const double* D3w, int* flags, cudaStream_t st);

}  // namespace wide
