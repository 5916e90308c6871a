/*
 * phx_abi.h -- C ABI of the B200 (sm_100a) scattering-rate library.
 *
 * Each entry point replaces one method of mir-group/phoebe's C++ call surface
 * for the 3-phonon / el-ph scattering-rate path; the reference method is
 * cited (file:line) beside each declaration.  Conventions:
 *   - every call returns int status (PHX_OK = 0); phx_last_error() gives text;
 *   - plain pointers and sizes only; "host" pointers are caller-owned host
 *     memory, "_d" pointers are device memory on the context's GPU;
 *   - arrays are C-order (row-major) in the reference's index order;
 *     complex arrays are interleaved (re, im) doubles;
 *   - eigenvector matrices are U[a][b]: row a = 3*atom + cartesian component
 *     (Wannier index for electrons), column b = band;
 *   - energies in Ry, lengths in Bohr, masses in Ry units, temperatures in Ry;
 *   - handles are not thread-safe; each context owns one CUDA stream.
 */
#ifndef PHX_ABI_H
#define PHX_ABI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PHX_OK 0
#define PHX_ERR_ARG 1      /* invalid argument or size */
#define PHX_ERR_CUDA 2     /* CUDA runtime error (message in phx_last_error) */
#define PHX_ERR_NOCONV 3   /* eigensolver hit its sweep cap */
#define PHX_ERR_STATE 4    /* call out of order (e.g. couplings before cache_d3) */
#define PHX_ERR_MESH 5     /* q1 +/- q2 not on the mesh */
#define PHX_ERR_NODEV 6    /* no CUDA device / extension unusable */

#define PHX_SMEAR_GAUSSIAN 0
#define PHX_SMEAR_ADAPTIVE 1

#define PHX_PREC_FP64 0        /* plain FP64 SIMT path */
#define PHX_PREC_SPLIT_BF16 1  /* BF16 hi+lo tcgen05 GEMM (8+8 mantissa bits), FP32 accumulate */
#define PHX_PREC_SPLIT_TF32 2  /* reserved: not built (rejected) */
#define PHX_PREC_SPLIT_FP16 3  /* FP16 hi+lo tcgen05 GEMM (11+11 mantissa bits; the FC3 operand
                                  scaled by a power of 2 per q2 chunk), FP32 accumulate */

typedef struct phx_ctx phx_ctx;
typedef struct phx_ph_h0 phx_ph_h0;
typedef struct phx_bands phx_bands;
typedef struct phx_v3 phx_v3;
typedef struct phx_el_h0 phx_el_h0;
typedef struct phx_elph phx_elph;
typedef struct phx_mlp phx_mlp;

/* ---- context ---------------------------------------------------------- */
/* Replaces initKokkos / DeviceManager (src/common_kokkos.cpp:104-134,182-190).
 * One CUDA stream per context; every call on a context runs on it.  Objects
 * (band structures, couplings, Hamiltonians) take their device memory from the
 * device's stream-ordered pool, whose release threshold phx_ctx_create raises
 * for this process.  phx_ctx_destroy releases the stream and the context's
 * buffers; objects created on it may still be destroyed afterwards, but no
 * other call may use it or them. */
int phx_ctx_create(int device, phx_ctx** out);
int phx_ctx_destroy(phx_ctx* ctx);
int phx_ctx_synchronize(phx_ctx* ctx);
/* Copies the last error message of this context (or of the library when
 * ctx is NULL) into buf; returns the status of the failing call. */
int phx_last_error(const phx_ctx* ctx, char* buf, size_t len);
/* Library version string (static storage). */
const char* phx_version(void);

/* ---- harmonic phonons (PhononH0) -------------------------------------- */
/* Host only, no GPU: acoustic sum rule "simple" + Wigner-Seitz reordering of
 * the QE force constants fc(3,3,n1,n2,n3,nat,nat) (Ry/Bohr^2).  cell is 3x3
 * with lattice vectors as columns, pos (nat,3).  Call with R = w = mat2R =
 * NULL to get numR; mat2R is written (numR, 3nat, 3nat).
 * Replaces PhononH0::setAcousticSumRule "simple" + reorderDynamicalMatrix +
 * wsInit (src/harmonic/phonon_h0_sum_rule.cpp:45-79;
 * src/harmonic/phonon_h0.cpp:426-535,672-771). */
int phx_ws_reorder(int nat, const double* cell, const double* pos, const int* grid,
                   const double* fc, int* numR, double* R, double* w, double* mat2R);

/* Builds the harmonic Hamiltonian on the GPU from QE force constants.
 * masses: per atom (Ry).  Replaces the PhononH0 constructor
 * (src/harmonic/phonon_h0.cpp:18-248; host->device copy :165-246). */
int phx_ph_h0_create(phx_ctx* ctx, int nat, const double* cell, const double* pos,
                     const double* masses, const int* grid, const double* fc,
                     phx_ph_h0** out);
int phx_ph_h0_destroy(phx_ph_h0* h0);
int phx_ph_h0_num_bands(const phx_ph_h0* h0);

/* Batched diagonalisation at nq Cartesian wavevectors (host buffers).
 * E (nq,nb); U (nq,nb,nb) complex; mass_scaling divides U by sqrt(m).
 * Replaces PhononH0::diagonalizeFromCoordinates (src/harmonic/phonon_h0.h:76-79)
 * and kokkosBatchedDiagonalizeFromCoordinates (src/harmonic/phonon_h0.h:106). */
int phx_ph_diag(phx_ph_h0* h0, int nq, const double* q_cart, int mass_scaling, double* E,
                double* U);

/* As phx_ph_diag plus group velocities vg (nq,nb,3) (Ry*Bohr) from the
 * finite-difference velocity operator with degenerate-subspace treatment.
 * U is mass-scaled.  Replaces kokkosBatchedDiagonalizeWithVelocities
 * (src/harmonic/phonon_h0.h:109) and PhononH0::diagonalizeVelocityFromCoordinates
 * (src/harmonic/phonon_h0.cpp:895-1070). */
int phx_ph_diag_velocities(phx_ph_h0* h0, int nq, const double* q_cart, double* E, double* U,
                           double* vg);

/* Device-resident band structure on a full Gamma-centred mesh (x fastest
 * point index, src/points.cpp:222-248).  Replaces PhononH0::populate /
 * ActiveBandStructure::builder for the phonon transport path
 * (src/harmonic/phonon_h0.cpp:389-394; src/bands/active_bandstructure.cpp:488-524). */
int phx_bands_create_mesh(phx_ph_h0* h0, const int* mesh, int with_velocities,
                          phx_bands** out);
/* Same, from caller-supplied host arrays (E (nq,nb), U (nq,nb,nb) complex
 * mass-scaled, vg (nq,nb,3) or NULL) -- FullBandStructure from another source. */
int phx_bands_create_from_host(phx_ctx* ctx, const int* mesh, const double* reciprocal_cell,
                               int nb, const double* E, const double* U, const double* vg,
                               phx_bands** out);
int phx_bands_destroy(phx_bands* b);
int phx_bands_num_points(const phx_bands* b);
/* Copy band data to host (any pointer may be NULL). */
int phx_bands_get(phx_bands* b, double* E, double* U, double* vg);

/* ---- 3-phonon vertex (Interaction3Ph) --------------------------------- */
/* D3 (nb,nb,nb,nr3,nr2) Ry/Bohr^3, R2 (nr2,3), R3 (nr3,3) Bohr,
 * w2 (nr2,nat,nat), w3 (nr3,nat,nat).  Replaces the Interaction3Ph
 * constructor (src/interaction/interaction_3ph.h:92-96; .cpp:5-68). */
int phx_v3_create(phx_ctx* ctx, int nat, int nr2, int nr3, const double* D3, const double* R2,
                  const double* R3, const double* w2, const double* w3, phx_v3** out);
int phx_v3_destroy(phx_v3* v3);
int phx_v3_set_precision(phx_v3* v3, int prec);
/* Interaction3Ph::cacheD3 (src/interaction/interaction_3ph.h:144; .cpp:100-175). */
int phx_v3_cache_d3(phx_v3* v3, const double* q2);
/* Interaction3Ph::getCouplingsSquared (src/interaction/interaction_3ph.h:128-138;
 * .cpp:179-405).  Eigenvectors are passed padded to nb columns:
 * ev1 (nq1,nb,nb), ev2 (nb,nb), ev3p/ev3m (nq1,nb,nb) complex, of which the
 * first nb1s[i] / nb2 / nb3ps[i] / nb3ms[i] columns are used.  Outputs are
 * ragged and concatenated: block i of outP holds (nb1s[i], nb2, nb3ps[i])
 * row-major at offset sum_{j<i} nb1s[j]*nb2*nb3ps[j] (likewise outM).
 * The precision of v3 applies: with a split precision the R3 transform of
 * the batch is one tensor-core GEMM (|V|^2 within 2e-6 (FP16) / 2e-5 (BF16)
 * of the batch's largest); nb <= 15 (one shared-memory block per q1). */
int phx_v3_couplings_sq(phx_v3* v3, int nq1, const double* q1s, const double* ev1,
                        const int* nb1s, const double* ev2, int nb2, const double* ev3p,
                        const int* nb3ps, const double* ev3m, const int* nb3ms, double* outP,
                        double* outM);
/* Interaction3Ph::estimateNumBatches (src/interaction/interaction_3ph.cpp:407-440),
 * against the GPU's free memory. */
int phx_v3_estimate_num_batches(phx_v3* v3, int nq1, int nb2, int* num_batches);

/* ---- scattering-rate builder (PhScatteringMatrix, linewidth mode) ------ */
typedef struct phx_lw_params {
  int num_temperatures;       /* nT <= 8 */
  const double* temperatures; /* (nT) Ry */
  int smearing;               /* PHX_SMEAR_* */
  double sigma;               /* Gaussian width (Ry) */
  int finalize;               /* 1: degeneracy-average row 0, zero excluded states */
  int q2_begin, q2_end;       /* q2 range to process ([0, nq) for the full builder) */
  /* Optional per-q1 window on q2 (no counterpart in the reference; uneven
   * work of the batched-instance workload): the pair (q1, q2) is counted only
   * when window_energy[q2] <= window_cut[q1].  Host arrays (nq), or both NULL
   * for every pair.  Runs on the FP64 path. */
  const double* window_energy;
  const double* window_cut;
  /* Isotope scattering (src/bte/ph_scattering.cpp:616-793): per atom the
   * reference's massVariance, i.e. the isotope mass variance of the species
   * times the atom's mass squared (Ry mass units); NULL disables it.  Adaptive
   * smearing takes the width from v1 and halves the delta, as the reference. */
  const double* isotope_coupling;
  /* Boundary scattering |v|/L n(n+1) (src/bte/ph_scattering.cpp:819-860),
   * added after the degeneracy averaging when finalize = 1; L in Bohr, <= 0
   * (or NaN) disables it. */
  double boundary_length;
} phx_lw_params;

typedef struct phx_lw_stats {
  double ms_total;            /* device time of the whole call */
  double ms_vertex;           /* device time of the q2 loop (R2 fold, conversions, pair kernels) */
  long long pairs;            /* (q1,q2) pairs processed */
  int kernel_launches;        /* kernels launched by the call */
  int pair_launches;          /* launches of the fused pair kernel */
  double ms_pair;             /* device time of those launches alone (CUDA events) */
  int plan_chunk, plan_slots; /* launch plan used (q2 per chunk, partial-sum slots) */
  int graph;                  /* 0 eager launches, 1 captured into a CUDA graph, 2 graph replayed */
  /* split path: the most near-cut-off events one pair launch recorded (their
   * adaptive deltas re-decided in FP64) and the capacity of the event list;
   * chunks of q2 with more events than that apply none of them and are re-run
   * in smaller pieces with the rates off (edge_overflow_chunks counts them) */
  long long edge_events_peak, edge_events_cap;
  int edge_overflow_chunks;
  /* phx_ph_linewidths_screened: vertices (q1, q2) the network dropped */
  long long pairs_screened_out;
  /* many-branch split builder: the tile shape in use (register tile of the
   * contractions, q1 planes per pass), tuned per problem shape; 0 elsewhere */
  int tile_rt, tile_qp;
} phx_lw_stats;

/* Whole PhScatteringMatrix::builder, switchCase 2 (linewidths), on the GPU:
 * symmetrizeCoupling, cutoffs, Gaussian/adaptive deltas, Bose factors,
 * accumulation, degeneracy averaging (src/bte/ph_scattering.cpp:60-935;
 * src/bte/scattering.cpp:1168-1318).  A_out (nT, nq*nb) host, the reference's
 * internalDiagonal (linewidth * n(n+1)).  stats may be NULL.  nb = 6 without
 * a q2 window runs on the fused kernels (FP64 or split precision); FP64 up to
 * nb = 16 or with a window on the shared-memory kernel; the split precisions
 * otherwise, and FP64 beyond 16 branches, on the many-branch builder (nb <= 48,
 * tcgen05 R3 transform, persistent work queue, tile shape tuned per problem). */
int phx_ph_linewidths(phx_v3* v3, phx_bands* bands, const phx_lw_params* params,
                      double* A_out, phx_lw_stats* stats);
/* Same with a device output buffer (nT*nq*nb doubles). */
int phx_ph_linewidths_d(phx_v3* v3, phx_bands* bands, const phx_lw_params* params,
                        double* A_out_d, phx_lw_stats* stats);

/* Linewidths with learned screening (no counterpart in the reference; the
 * screened builder that the north star's learned part asks for).  The
 * network net (phx_mlp_create with 12 inputs) predicts, for every vertex
 * (q1, q2) of the q2 range, log10 of the largest fraction that the vertex
 * adds to the linewidth of any mode of q1 (its "+" process of (q1, q2) and
 * "-" process of (q1, -q2), the builder's unit of work).  Vertices predicted
 * below log10_threshold are dropped; every other one is evaluated exactly on
 * the many-branch builder in the precision of v3.  Inputs of a vertex: the
 * fractional coordinates of q1, q2 and q3 = q1 + q2, and the lowest phonon
 * energy of each over the largest of the mesh (screening.pair_features).
 * stats->pairs_screened_out counts the dropped vertices.  A_out host. */
int phx_ph_linewidths_screened(phx_v3* v3, phx_bands* bands, const phx_lw_params* params, phx_mlp* net,
                               double log10_threshold, double* A_out, phx_lw_stats* stats);

/* ---- scattering-matrix modes of the builder (nb = 6, no q2 window) ----
 * Both precisions of the coupling object: PHX_PREC_FP64, or the split paths,
 * whose matrix elements are within 1e-6 of the largest FP64 element (their
 * sums over q2 within the linewidths' 1e-5).  The stored matrix is FP64.
 * States are numbered s = iq * nb + ib (the reference's BteIndex without
 * symmetries).  The rates, cut-offs, exclusions and time-reversal pairing are
 * those of phx_ph_linewidths; the differences are the reference's: the
 * diagonal is the linewidth x n(n+1) WITHOUT degeneracy averaging, plus
 * boundary scattering; off-diagonal elements are the sums over b3 of the "+"
 * rates minus the two "-" rates (and minus the isotope rates) of each pair of
 * states.  With finalize = 0 the diagonal is not written and no exclusion is
 * applied (partial sums of a q2 slice). */
typedef struct phx_smatrix phx_smatrix;

/* PhScatteringMatrix::builder with switchCase 0 (scatteringMatrixInMemory,
 * src/bte/ph_scattering.cpp:382-406,520-547,714-738,846-847,864-890,910-933;
 * src/bte/scattering.cpp:105-160): the whole matrix, ns x ns FP64, kept in
 * device memory by the handle (18.4 GB for the 20x20x20 diamond mesh).  One
 * temperature, as the reference requires.  Fails with PHX_ERR_ARG when the
 * matrix does not fit in free device memory. */
int phx_ph_smatrix_create(phx_v3* v3, phx_bands* bands, const phx_lw_params* params, phx_smatrix** out,
                          phx_lw_stats* stats);
int phx_smatrix_num_states(const phx_smatrix* m);
/* internalDiagonal (ns) of the stored matrix (ScatteringMatrix::diagonal, scattering.cpp:165-178) */
int phx_smatrix_diagonal(phx_smatrix* m, double* diag);
/* rows row0 .. row0+nrows-1 of A, row-major (nrows, ns) host (theMatrix(row, col)) */
int phx_smatrix_get_rows(phx_smatrix* m, int row0, int nrows, double* out);
/* ScatteringMatrix::dot (off_diagonal = 0: rows and columns of excluded states
 * left out, scattering.cpp:266-330) or offDiagonalDot (off_diagonal = 1: the
 * diagonal left out, :180-232) of the stored matrix: y = A x for nvec vectors,
 * x and y (nvec, 3, ns) host. */
int phx_smatrix_dot(phx_smatrix* m, int nvec, const double* x, int off_diagonal, double* y);
/* Same with device vectors; ms (may be NULL): device time of the product. */
int phx_smatrix_dot_d(phx_smatrix* m, int nvec, const double* x_d, int off_diagonal, double* y_d, float* ms);
/* A -> (A + A^T) / 2 in place (ScatteringMatrix::symmetrize, src/bte/scattering.cpp:1149-1166;
 * the reference's symmetrizeMatrix option before its exact solvers). */
int phx_smatrix_symmetrize(phx_smatrix* m);
/* Relaxons (src/apps/phonon_transport_app.cpp:386-420).
 * ScatteringMatrix::a2Omega (src/bte/scattering.cpp:366-434): in place,
 * A(i, j) /= sqrt(n_i(n_i+1) n_j(n_j+1)) for included states i, j, and the
 * diagonal returned by phx_smatrix_diagonal /= n_i(n_i+1).  A second call does
 * nothing.  Products (phx_smatrix_dot) are refused afterwards (PHX_ERR_STATE). */
int phx_smatrix_a2omega(phx_smatrix* m);
/* ScatteringMatrix::diagonalize (scattering.cpp:872-910; ParallelMatrix
 * ::diagonalize, src/algebra/PMatrix.cpp:99-160 and 266-404): eigenvalues and
 * eigenvectors of the symmetric matrix read from its UPPER triangle (uplo 'U'),
 * computed in place: as in the reference, the matrix is destroyed.
 * num_eigenvalues <= 0 or = ns: all of them; else the smallest num_eigenvalues.
 * eigenvalues: (ns) host, ascending; *num_found: how many were computed.
 * Afterwards phx_smatrix_get_rows returns rows of the eigenvector matrix
 * Theta(s, alpha), columns alpha < *num_found.  More eigenvalues than states:
 * PHX_ERR_ARG; a solver failure to converge: PHX_ERR_NOCONV. */
int phx_smatrix_diagonalize(phx_smatrix* m, int num_eigenvalues, double* eigenvalues, int* num_found);
/* The relaxon-basis solve of PhononThermalConductivity::calcFromRelaxons
 * without symmetries (src/observable/phonon_thermal_cond.cpp:316-380):
 * y = Theta diag(g) Theta^T x, g_alpha = 1/lambda_alpha for the computed
 * eigenvalues lambda_alpha > 0 and 0 otherwise; x and y (nvec, 3, ns) host.
 * With x = dn/dT v / sqrt(n(n+1)) this gives the relaxon population before
 * the reference's final sqrt(n(n+1)) rescaling. */
int phx_smatrix_relaxon_solve(phx_smatrix* m, int nvec, const double* x, double* y);
int phx_smatrix_destroy(phx_smatrix* m);

/* PhScatteringMatrix::builder with switchCase 1 (ScatteringMatrix::dot when the
 * matrix is not stored, src/bte/ph_scattering.cpp:408-431,549-572,741-759,
 * 849-855,891-897): y = A x for nvec vectors, one matrix per temperature,
 * x and y (nvec, nT, 3, ns) host, in one builder pass without storing A. */
int phx_ph_smatrix_dot(phx_v3* v3, phx_bands* bands, const phx_lw_params* params, int nvec, const double* x,
                       double* y, phx_lw_stats* stats);
/* Same with device vectors. */
int phx_ph_smatrix_dot_d(phx_v3* v3, phx_bands* bands, const phx_lw_params* params, int nvec,
                         const double* x_d, double* y_d, phx_lw_stats* stats);

/* Allocation-free variant of phx_ph_linewidths_d (no counterpart in the
 * reference).  For callers that cannot allocate device memory when they call
 * the builder -- e.g. an application that has given all free device memory
 * to its own pool allocator, or one that must not pay cudaMalloc/cudaFree's
 * implicit device synchronisation inside a latency-critical loop.  It calls
 * no cudaMalloc/cudaFree: the plain FP64 path runs with every intermediate
 * buffer in a 16 MiB array that the library reserves statically on each GPU
 * where it is loaded (held until the process exits).  The caller passes the
 * device output A_out_d (nT*nq*nb doubles).  Limit: Bose table and partial
 * sums, 16*nq*nb*nT bytes, plus one q2 slab of the cached vertex,
 * 16*nr3*nb^3 bytes, must fit in 16 MiB; larger problems are rejected with
 * PHX_ERR_ARG.  The first call on a device (and in each new CUDA context of
 * it) looks up the array's address with cudaGetSymbolAddress.  Never call
 * this function inside a stream capture: every call sets kernel attributes,
 * copies the temperatures from pageable host memory and synchronises the
 * stream before it returns.  All calls share the array and leave their
 * contents in it (the call clears what must start at zero): calls that
 * overlap on the same GPU race.  The precision setting of v3 is ignored
 * (FP64).  Returns after the stream has drained. */
int phx_ph_linewidths_static(phx_v3* v3, phx_bands* bands, const phx_lw_params* params,
                             double* A_out_d);

/* RTA thermal conductivity (atomic units; x thConductivityAuToSi for W/m/K)
 * from A_out: tau = n(n+1)/A_out, kappa_ij = sum dn/dT v_i tau v_j E/(Nq V).
 * kappa (nT,3,3) host.  Replaces BulkTDrift + getSingleModeTimes +
 * PhononThermalConductivity::calcFromPopulation (src/bte/drift.cpp:3-29;
 * src/bte/scattering.cpp:484-527; src/observable/phonon_thermal_cond.cpp:64-113). */
int phx_ph_rta_kappa(phx_bands* bands, int nT, const double* temperatures,
                     const double* A_out, double volume, double* kappa);

/* ---- electronic Wannier Hamiltonian (ElectronH0Wannier) ----------------- */
/* Build from the Wannier Hamiltonian H(R) (nR,nw,nw) complex (Ry) on the
 * Bravais vectors R (nR,3) Bohr with degeneracies deg (nR); cell as in
 * phx_ph_h0_create.  Replaces the ElectronH0Wannier constructor without
 * shifted vectors (src/harmonic/electron_h0_wannier.cpp:6-60). */
int phx_el_h0_create(phx_ctx* ctx, int nw, int nR, const double* cell, const double* R,
                     const double* deg, const double* H, phx_el_h0** out);
int phx_el_h0_destroy(phx_el_h0* h);
int phx_el_h0_num_bands(const phx_el_h0* h);
/* H(k) = sum_R e^{+i k.R}/deg_R H(R), ascending energies E (nk,nw), eigenvectors
 * U (nk,nw,nw) complex with U[w][b] = component w of band b, and, when vg is
 * not NULL, group velocities (nk,nw,3) of the Hellmann-Feynman operator with
 * degenerate subspaces (1 micro-eV) rediagonalised and zero at Gamma.
 * Replaces batchedDiagonalizeFromCoordinates / batchedDiagonalizeWithVelocities
 * (src/harmonic/electron_h0_wannier.cpp:160-235,633-760; Kokkos :777-999). */
int phx_el_diag(phx_el_h0* h, int nk, const double* k, double* E, double* U, double* vg);
/* Device band structure of a Gamma-centred k mesh (ElectronH0Wannier::populate,
 * src/harmonic/electron_h0_wannier.h:91-114). */
int phx_el_bands_create_mesh(phx_el_h0* h, const int* mesh, int with_velocities, phx_bands** out);

/* ---- electron-phonon coupling (InteractionElPhWan) ---------------------- */
/* Upload the Wannier-basis coupling g(Re, Rp, nu, w1, w2), complex FP32
 * (nRe,nRp,nph,nw,nw), with the electronic and phononic Bravais vectors (Bohr)
 * and their degeneracies.  Replaces the InteractionElPhWan constructor
 * (src/interaction/interaction_elph.h:89-120; layout of :45-47). */
int phx_elph_create(phx_ctx* ctx, int nw, int nph, int nRe, int nRp, const double* Re,
                    const double* degE, const double* Rp, const double* degP, const float* g,
                    phx_elph** out);
int phx_elph_destroy(phx_elph* e);
/* cacheElPh (src/interaction/interaction_elph.cpp:492-701): transform over Re
 * at k1 (e^{+i k1.Re}/deg) and rotate by the k1 eigenvectors U1 (nw,nb1)
 * complex; the result stays on the device for phx_elph_couplings_sq. */
int phx_elph_cache_k1(phx_elph* e, const double* k1, const double* U1, int nb1);
/* calcCouplingSquared + getCouplingSquared (src/interaction/interaction_elph.cpp:229-448,
 * no polar correction): for nk2 final states with phonon wavevectors q3 (nk2,3),
 * electron eigenvectors U2s (nk2,nw,nb2max) complex (first nb2s[i] columns used)
 * and phonon eigenvectors ev3s (nk2,nph,nph) complex U[a][nu], writes
 * coupling (nk2,nb1,nb2max,nph) = |g(b1,b2,nu)|^2 (zero beyond nb2s[i]). */
int phx_elph_couplings_sq(phx_elph* e, int nk2, const double* q3, const double* U2s, const int* nb2s,
                          int nb2max, const double* ev3s, double* coupling);

/* Precision of the Re and Rp transforms inside phx_el_linewidths (the first steps
 * of cacheElPh and calcCouplingSquared, interaction_elph.cpp:540-580,364-374):
 * PHX_PREC_FP64 (default) or PHX_PREC_SPLIT_BF16 (tcgen05 BF16 hi+lo; the Re
 * transform adds its 64-deep chunk sums in FP64, the Rp transform accumulates in
 * FP32).  The U1 rotation, the phonon and U2 rotations, |g|^2 and the rates stay
 * FP64.  The first split call builds a BF16 image of the coupling tensor (as large
 * as the FP32 tensor), kept until phx_elph_destroy. */
int phx_elph_set_precision(phx_elph* e, int precision);

typedef struct phx_el_params {
  int num_temperatures;       /* <= 4 */
  const double* temperatures; /* Ry */
  double chemical_potential;  /* Ry */
  double window;              /* half width (Ry) of the active window around mu */
  int smearing;               /* PHX_SMEAR_GAUSSIAN / PHX_SMEAR_ADAPTIVE */
  double sigma;               /* Gaussian width (Ry) */
  double norm;                /* prefactor of every rate (1/N of the summed q mesh) */
  int num_k1;                 /* outer k points */
  const int* k1_list;         /* their k-mesh indices (host) */
} phx_el_params;

/* ElScatteringMatrix::builder, linewidth mode (src/bte/el_scattering.cpp:38-405),
 * for the outer k points k1_list of the electron mesh el_bands, every q of the
 * phonon mesh ph_bands (the q mesh must divide the k mesh) and k2 = k1 + q:
 * states outside |E - mu| <= window are inactive; rates
 * |g|^2 ((f2 + n3) d(E1-E2+w3) + (1 - f2 + n3) d(E1-E2-w3)) norm pi / w3 with
 * w3 >= 5 cm^-1, |g|^2 symmetrised over degenerate blocks, then degeneracy
 * averaging of temperature row 0.  out (nT, num_k1, nw) host, zero for
 * inactive states.  stats may be NULL. */
int phx_el_linewidths(phx_elph* e, phx_bands* el_bands, phx_bands* ph_bands,
                      const phx_el_params* params, double* out, phx_lw_stats* stats);

/* ---- learned screening network (no counterpart in the reference) -------- */
/* MLP nin -> hidden (x depth, GELU) -> 1 with parameters laid out per layer as
 * W (nout,nin) row-major then b (nout), FP32 master copies; every product uses
 * the weights rounded to BF16 with FP32 accumulation.  params may be NULL
 * (uninitialised).  Kernels: tiled GEMM forward/backward, GELU, MSE, Adam. */
int phx_mlp_create(phx_ctx* ctx, int nin, int hidden, int depth, const float* params, phx_mlp** out);
int phx_mlp_destroy(phx_mlp* net);
long long phx_mlp_num_params(const phx_mlp* net);
int phx_mlp_get_params(phx_mlp* net, float* params);
int phx_mlp_set_params(phx_mlp* net, const float* params);
/* y (B) = net(X (B,nin)), host arrays */
int phx_mlp_infer(phx_mlp* net, int B, const float* X, float* y);
/* gradient (num_params) of the mean squared error mean_b (net(X_b) - t_b)^2, and the loss */
int phx_mlp_grad(phx_mlp* net, int B, const float* X, const float* t, float* grad, float* loss);
/* Adam (beta 0.9/0.999, eps 1e-8) on shuffled mini-batches for the given epochs;
 * loss_per_epoch (epochs) may be NULL. */
int phx_mlp_train(phx_mlp* net, int n, const float* X, const float* t, int epochs, int batch, float lr,
                  unsigned long long seed, float* loss_per_epoch);

/* ---- diagnostics -------------------------------------------------------- */
/* Self-test of the split-precision tensor-core GEMM used by the builder: one
 * 128 x N tile C = A * B^T with A (128,Kp) and B (N,Kp) FP32 host arrays,
 * split into BF16 hi+lo and accumulated as hi*hi + hi*lo + lo*hi in FP32 via
 * tcgen05.mma with the builder's shared-memory layouts.  No reference
 * counterpart (validates this library's own tensor-core building block). */
int phx_diag_tc_gemm(phx_ctx* ctx, int N, int Kp, const float* A, const float* B, float* C);

/* Test hook (no reference counterpart): capacity of the split path's
 * near-cut-off event list per pair launch, for this process (0: the default,
 * 2^18).  A linewidth chunk with more events is re-run in pieces whose events
 * fit, so the results do not depend on it; a small capacity exercises that
 * path.  The matrix modes fail with PHX_ERR_ARG on an overflow. */
int phx_debug_set_split_edge_cap(unsigned cap);

#ifdef __cplusplus
}
#endif
#endif /* PHX_ABI_H */
