/*
 * integral_gpu.h — C ABI of the B200 (sm_100a) two-electron integral path.
 *
 * Drop-in boundary for the Rust crate `integral` (nmrtist/integral 0.4.3):
 * the crate's C-ABI crate `integral-sys` exports only
 * `integral_abi_version()` (crates/integral-sys/src/lib.rs:21); the entry
 * points below extend that seam with the GPU-backed two-electron path so the
 * Rust host (Basis, EriBuilder, DirectContractor, DirectGradContractor) can
 * call CUDA through plain pointers and sizes.  Every entry point returns an
 * int status (IGPU_OK = 0, negative = error, never unwinds); the message of
 * the last failure on the calling thread is igpu_last_error_string().
 *
 * Layouts follow the reference exactly:
 *   - AO order = shell order, n_func per shell (Cartesian (l+1)(l+2)/2 in
 *     src/math/am.rs order, spherical 2l+1 in solid_harmonics::m_order order);
 *   - dense ERI: eri[((i*nao + j)*nao + k)*nao + l] (src/integrals.rs:646-654);
 *   - densities / J / K: row-major nao x nao, ndens of them back to back;
 *   - gradient: dE/dR (not force), natom x 3, atoms in Basis::atoms() order
 *     (first appearance of a bitwise-equal centre, src/shell.rs:250-258).
 * Outputs of igpu_jk*, igpu_grad* ACCUMULATE (+=) into the caller's buffers
 * (src/direct.rs:398-403, src/direct_grad.rs:476-484); igpu_eri_dense and
 * igpu_eri_builder_fill ASSIGN.
 */
#ifndef INTEGRAL_GPU_H
#define INTEGRAL_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IGPU_ABI_VERSION 1u

/* status codes (IntegralError variants of src/lib.rs:83-118 plus the
 * misuse panics of src/direct.rs:141-159 / src/direct_grad.rs:337-346) */
#define IGPU_OK 0
#define IGPU_ERR_INVALID_ARGUMENT (-1)
#define IGPU_ERR_EMPTY_CONTRACTION (-2)       /* IntegralError::EmptyContraction */
#define IGPU_ERR_MISMATCHED_CONTRACTION (-3)  /* IntegralError::MismatchedContraction */
#define IGPU_ERR_ANGULAR_MOMENTUM (-4)        /* IntegralError::AngularMomentumTooHigh */
#define IGPU_ERR_ANGULAR_MOMENTUM_GRAD (-5)   /* ...TooHighForGradient */
#define IGPU_ERR_DENSITY_COUNT (-6)           /* 1..64 densities (direct.rs:141-148) */
#define IGPU_ERR_LENGTH (-7)                  /* buffer length mismatch */
#define IGPU_ERR_NONCANONICAL_BRA (-8)        /* bra pair index out of range */
#define IGPU_ERR_CUDA (-9)
#define IGPU_ERR_OUT_OF_MEMORY (-10)
#define IGPU_ERR_UNSUPPORTED (-11)            /* class not built for the GPU */
#define IGPU_ERR_NO_DEVICE (-12)

/* Engine (src/integrals.rs:329-338).  The GPU evaluates every quartet by Rys
 * quadrature; the value is kept so the plan reports what the host asked for. */
#define IGPU_ENGINE_AUTO 0
#define IGPU_ENGINE_OSHGP 1
#define IGPU_ENGINE_RYS 2

/* Arithmetic of the quartet kernels.  FP64: every quartet in double.
 * MIXED: quartets whose Schwarz estimate Q_ij*Q_kl*M is below the plan's
 * cutoff run in FP32 (Rys roots, recurrences, primitive contraction and, for
 * J/K, the horizontal recurrences, spherical transform and density
 * contraction against an FP32 copy of the densities), the rest in FP64; M is
 * max|D| (or the term matrices' maximum) rounded up to a power of two, so
 * densities whose maxima share a binade share one task list.  All
 * J/K/gradient accumulation is FP64. */
#define IGPU_PRECISION_FP64 0
#define IGPU_PRECISION_MIXED 1

typedef struct igpu_plan igpu_plan;

/* One contracted shell (src/shell.rs:49-55): raw contraction coefficients;
 * the plan applies the per-primitive normalisation (shell.rs:182-187). */
typedef struct {
  int l;
  int spherical; /* 0 Cartesian, 1 real spherical */
  double center[3];
  int nprim;
  const double* exps;
  const double* coefs;
} igpu_shell;

/* One product term factor * left (x) right of a two-particle density
 * (GradDensityTerm, src/direct_grad.rs:21-25); left/right symmetric nao x nao. */
typedef struct {
  double factor;
  const double* left;
  const double* right;
} igpu_term;

/* Counters of the last J/K or gradient call on a plan. */
typedef struct {
  uint64_t quartets;          /* canonical shell quartets that survived screening */
  uint64_t quartet_hash;      /* order-independent fingerprint of that list */
  uint64_t quartets_fp32;     /* of them, evaluated in FP32 (MIXED) */
  uint64_t prim_quartets;     /* surviving primitive quartets */
  double model_flops;         /* fixed Rys flop model of the surviving work */
  double kernel_ms;           /* device time of the quartet kernels */
  uint32_t launches;          /* kernels launched by the call */
} igpu_stats;

/* One quartet-kernel launch of the last J/K or gradient call. */
typedef struct {
  int la, lb, lc, ld;         /* angular class in evaluation orientation */
  int fp32;                   /* evaluated in FP32 */
  int team;                   /* lanes per quartet */
  uint32_t grid;              /* blocks of 128 threads */
  uint64_t tasks;             /* quartets in the launch's task list */
  uint64_t quartets;          /* of them accepted by the screening */
  uint64_t prim_quartets;
  double ms;                  /* device time (CUDA events) */
  double model_flops;         /* fixed Rys flop model of the accepted work */
  uint32_t chunk;             /* tasks a warp claims per grab */
  uint32_t reserved;
} igpu_launch_record;

/* integral-sys `integral_abi_version` (crates/integral-sys/src/lib.rs:21). */
uint32_t igpu_abi_version(void);

const char* igpu_last_error_string(void);

/* Plan = DirectContractor::with_engine / DirectGradContractor::with_engine /
 * EriBuilder::with_engine precompute (src/direct.rs:59-87,
 * src/direct_grad.rs:180-247, src/eri_builder.rs:238-270): shells, offsets,
 * effective coefficients, c2s, canonical pairs, primitive-pair data and the
 * Schwarz bounds (computed on the device once, at creation). */
int igpu_plan_create(const igpu_shell* shells, size_t nsh, int engine, igpu_plan** out);
int igpu_plan_destroy(igpu_plan* plan);
/* Basis::nao (shell.rs:160), Basis::atoms().len(), bra_pairs().len(), nsh. */
int igpu_plan_query(const igpu_plan* plan, size_t* nao, size_t* natom, size_t* nbra, size_t* nsh);
/* DirectContractor::bra_pairs (direct.rs:95): canonical (i, j), i >= j,
 * row-major; pairs[2p] = i, pairs[2p+1] = j. */
int igpu_bra_pairs(const igpu_plan* plan, uint32_t* pairs);
/* Basis::atoms (shell.rs:250-258): natom x 3 centres. */
int igpu_atoms(const igpu_plan* plan, double* xyz);
/* Basis::schwarz_bounds (integrals.rs:835-862): nsh x nsh, row-major.
 * Wherever the reference's Auto policy (integrals.rs:374-388) evaluates a
 * diagonal quartet with OS/HGP, which covers every shell pair of a basis of
 * contracted shells, the plan holds a bit-exact evaluation of it (run on the
 * device with the reference's order of operations and no fused
 * multiply-adds), so the screened quartet lists equal the reference's by
 * construction; the other pairs (see igpu_schwarz_bounds) keep the device's
 * Rys evaluation.  Molecule batches hold the same bounds. */
int igpu_schwarz(const igpu_plan* plan, double* q);
/* Basis::schwarz_bounds of a shell list on the host, without a device or a
 * plan: the same bit-exact bounds, nsh x nsh row-major.  An ordered shell
 * pair whose diagonal quartet the Auto policy sends to the Rys engine (one
 * primitive on each shell at l_i + l_j >= 3, fewer than four primitive pairs
 * at l_i + l_j >= 7, or l_i + l_j > 8) has no host evaluation: its entry is
 * NaN and it is counted in *n_rys (n_rys may be NULL).  A plan holds the
 * device evaluation for those pairs (within 1e-14 of the reference). */
int igpu_schwarz_bounds(const igpu_shell* shells, size_t nsh, double* q, size_t* n_rys);
/* Plan cutoff for IGPU_PRECISION_MIXED (default 1e-3). */
int igpu_set_mixed_cutoff(igpu_plan* plan, double cutoff);
/* Primitive screen of the FP32 quartets of IGPU_PRECISION_MIXED J/K (no
 * counterpart in the reference, which evaluates every primitive quartet that
 * survives its 1e-32 pair screen): inside an FP32 quartet, a primitive
 * quartet whose magnitude bound |E_ab E_cd| 2 pi^{5/2} / (p q sqrt(p + q))
 * times max|D| is below eps is skipped (default 1e-15).  0 evaluates every
 * primitive quartet; the FP64 path never skips one. */
int igpu_set_mixed_prim_cutoff(igpu_plan* plan, double eps);
/* The plan's two mixed-precision cutoffs (either pointer may be NULL). */
int igpu_get_mixed_cutoffs(const igpu_plan* plan, double* cutoff, double* prim_eps);
/* EriKernel (src/integrals.rs:304-321) of every later call on the plan:
 * omega = 0 is Coulomb 1/r (the default); omega > 0 finite is the long-range
 * erf(omega r)/r (Basis::eri_kernel, EriBuilder::kernel, the gradient's
 * kernel argument).  The J/K entries apply it too, with no counterpart in
 * the reference (its DirectContractor is Coulomb only).  Screening keeps the
 * Coulomb Schwarz bounds, which bound the attenuated integrals.  Any other
 * omega is IGPU_ERR_INVALID_ARGUMENT (the reference's check_erf_omega). */
int igpu_set_erf_omega(igpu_plan* plan, double omega);

/* Basis::eri / eri_with (integrals.rs:664-754): dense nao^4 tensor into a
 * host buffer of nao^4 doubles (assigned). */
int igpu_eri_dense(igpu_plan* plan, double* out);
/* EriBuilder::partition + fill (eri_builder.rs:337-417) for the canonical
 * bra pairs in `bra_subset` (NULL = all): every (ij|kl) over all canonical
 * ket pairs scattered into the 4 bra/ket-internal slots of the host nao^4
 * buffer (assigned; other elements untouched). */
int igpu_eri_builder_fill(igpu_plan* plan, const uint32_t* bra_subset, size_t nsub, double* out);
/* Basis::eri_screened (src/integrals.rs:864-981): the dense tensor with
 * every canonical quartet of Q_ij*Q_kl < tau left zero in all its
 * permutation slots; *total and *skipped (either may be NULL) receive the
 * ScreeningStats counts of canonical quartets.  NaN tau is rejected. */
int igpu_eri_screened(igpu_plan* plan, double tau, double* out, uint64_t* total, uint64_t* skipped);
/* Basis::eri_block (src/integrals.rs:600-640): the (ij|kl) block of shells
 * i, j, k, l in that order, row-major [n_i][n_j][n_k][n_l] over the shells'
 * functions; out holds n_i*n_j*n_k*n_l doubles (host). */
int igpu_eri_block(igpu_plan* plan, int i, int j, int k, int l, double* out);
/* PackedEriBuilder::build / fill (src/packed_eri.rs:156-237): the
 * symmetry-unique tensor, AO pairs numbered shell-pair blocked (canonical
 * shell pair, then (a, b) row-major with b <= a on diagonal pairs, see
 * packed_eri.rs:10-21), element (t|u), u <= t, at t(t+1)/2 + u; m(m+1)/2
 * doubles for m = nao(nao+1)/2.  Writes every canonical quartet with a bra
 * in bra_subset (all when NULL) into `out` (host, caller-initialised; other
 * elements are left as they are).  threshold > 0 skips quartets with
 * Q_ij*Q_kl < threshold; threshold <= 0 screens nothing. */
int igpu_eri_packed(igpu_plan* plan, double threshold, const uint32_t* bra_subset, size_t nsub, double* out);

/* Density fitting (src/df.rs).  An auxiliary basis is attached to a plan
 * (Eri3cBuilder::new(main, aux), df.rs:354-383); each aux shell is paired
 * with the unit s dummy (one zero-exponent primitive of coefficient 1,
 * df.rs:33-38), so (mu nu|P) = (mu nu|P 1s) and (P|Q) = (P 1s|Q 1s) run on the
 * four-centre kernels.  Attaching again replaces the earlier aux basis; the
 * main-basis entries are unaffected.  Aux shells are validated like main
 * shells; l above the compiled GPU classes is IGPU_ERR_UNSUPPORTED.  The
 * aux Schwarz factors are evaluated on the device here. */
int igpu_plan_attach_aux(igpu_plan* plan, const igpu_shell* aux, size_t naux_shells);
/* naux (aux functions) and the aux shell count of the attached basis. */
int igpu_aux_query(const igpu_plan* plan, size_t* naux, size_t* naux_shells);
/* Basis::schwarz_aux_bounds (df.rs:250-286): QP[p] = sqrt(max_mu (mu|mu))
 * over the (p|p) block, one per aux shell. */
int igpu_schwarz_aux(const igpu_plan* plan, double* qp);
/* Basis::eri_2c / eri_2c_kernel (df.rs:49-145) over the attached aux basis:
 * row-major naux x naux, exactly symmetric. */
int igpu_eri_2c(igpu_plan* plan, double* out);
/* Eri3cBuilder::build / fill / fill_filtered (df.rs:463-520): (mu nu|P) at
 * out[(mu*nao + nu)*naux + P] for the canonical main bra pairs in bra_subset
 * (all when NULL), both the (i, j) and (j, i) bands, over the aux shells p
 * with keep[p] != 0 (all when keep is NULL).  `out` is the host buffer of
 * nao*nao*naux doubles; slots of other bras and of skipped aux shells keep
 * their content. */
int igpu_eri_3c(igpu_plan* plan, const uint32_t* bra_subset, size_t nsub, const uint8_t* keep, double* out);

/* DirectContractor::density_shell_bounds (direct.rs:103-125): per density the
 * max |D| of every ordered shell block, ndens x nsh x nsh. */
int igpu_density_shell_bounds(const igpu_plan* plan, const double* dens, int ndens, double* bounds);

/* DirectContractor::accumulate_bra_pair (direct.rs:131-218) over the
 * canonical bra pairs in bra_subset (NULL = all) in one launch sequence:
 * J[d] += sum (ab|cd) D[d]_cd, K[d] += sum (ab|cd) D[d]_bd over the
 * Schwarz/density-screened canonical quartets.  Host buffers; K may be NULL
 * when want_k == 0.  The subset's indices must be distinct (a repeat is
 * IGPU_ERR_INVALID_ARGUMENT: it would count once here, twice through
 * per-bra calls); the gradient entries below follow the same rule. */
int igpu_jk(igpu_plan* plan, const double* dens, int ndens, const uint32_t* bra_subset, size_t nsub,
            double threshold, int want_k, int precision, double* J, double* K);
/* Same with device-resident D, J, K on a caller stream (cudaStream_t). */
int igpu_jk_device(igpu_plan* plan, const double* d_dens, int ndens, const uint32_t* bra_subset,
                   size_t nsub, double threshold, int want_k, int precision, double* d_J,
                   double* d_K, void* stream);

/* igpu_jk_device without any device allocation.  It has no counterpart in
 * the reference.  It is for callers that may not call cudaMalloc/cudaFree
 * while they run: an SCF driver whose device memory is all handed out by
 * its own pool allocator, or a pipeline in which cudaFree's implicit device
 * synchronisation would stall other streams.  FP64, every canonical bra
 * pair, J += and K += directly (any density, symmetric or not).
 * Its scratch lives in file-scope device arrays that every GPU loading this
 * library holds until the process exits: team scratch 64 MiB, density
 * bounds ndens * nsh^2 <= 2^21 doubles, 1024 work counters.  A request
 * beyond those sizes returns IGPU_ERR_UNSUPPORTED with a message.  The
 * first call on a device looks up the arrays' device addresses (set-up);
 * make that first call before any stream capture.  Every call shares the
 * arrays, so calls that overlap on the GPU race: order them on one stream.
 * Also needs the FP64 task list of `threshold`, built by one earlier
 * igpu_jk or igpu_jk_device call on this plan with the same threshold.
 * The plan's device must be the current device.  With a caller stream the
 * call only queues its work on that stream (read J/K after synchronising
 * it); with stream == NULL it runs on the plan's stream and returns when
 * the work is done.  Does not update igpu_last_stats / igpu_last_profile. */
int igpu_jk_device_static(igpu_plan* plan, const double* d_dens, int ndens, double threshold, int want_k,
                          double* d_J, double* d_K, void* stream);

/* DirectGradContractor::density + accumulate_bra_pair / contract
 * (direct_grad.rs:272-392): out[natom][3] += dE/dR.  Host buffers. */
int igpu_grad(igpu_plan* plan, const igpu_term* coulomb, int ncoul, const igpu_term* exchange,
              int nexch, const uint32_t* bra_subset, size_t nsub, double threshold, int precision,
              double* out);
/* Same with device-resident term matrices and output on a caller stream. */
int igpu_grad_device(igpu_plan* plan, const igpu_term* d_coulomb, int ncoul,
                     const igpu_term* d_exchange, int nexch, const uint32_t* bra_subset,
                     size_t nsub, double threshold, int precision, double* d_out, void* stream);

/* Molecule batches (no counterpart in the reference, whose callers loop
 * over one DirectContractor / DirectGradContractor per molecule,
 * src/direct.rs:19-21, src/direct_grad.rs:140-142).  A batch holds many
 * independent molecules of uneven size: molecule m has mol_nsh[m] shells,
 * consecutive in `shells`.  Each step runs, for every molecule, one direct
 * J/K build with its own density and, optionally, the density-direct
 * gradient of E = coul_factor * tr(D J[D])-type and exch_factor *
 * tr(D K[D])-type terms (GradDensityTerm (coul_factor, D, D) and
 * (exch_factor, D, D)), with exactly the screening, integrals and
 * contractions of a plan of that molecule alone.  Every angular class of
 * every molecule runs in one persistent launch per class; the first step
 * with a given (threshold, precision split, want_k, want_grad, factors,
 * density symmetry) captures the whole sequence into a CUDA graph, later
 * steps replay it. */
typedef struct igpu_batch igpu_batch;
int igpu_batch_create(const igpu_shell* shells, const size_t* mol_nsh, size_t nmol, igpu_batch** out);
int igpu_batch_destroy(igpu_batch* batch);
/* nao, natom (bitwise-equal centres inside the molecule) and nsh of molecule `mol`. */
int igpu_batch_query(const igpu_batch* batch, size_t mol, size_t* nao, size_t* natom, size_t* nsh);
/* One step over host buffers.  dens, J and K hold the molecules' nao_m x
 * nao_m matrices back to back (row-major); grad holds natom_m x 3 per
 * molecule back to back (dE/dR).  J, K and grad accumulate (+=).  stats
 * (may be NULL) receives the step's counters: kernel_ms is the device time
 * of the graph launch, launches the kernels it ran. */
int igpu_batch_jk_grad(igpu_batch* batch, const double* dens, double threshold, int precision, int want_k,
                       int want_grad, double coul_factor, double exch_factor, double* J, double* K, double* grad,
                       igpu_stats* stats);
int igpu_batch_set_mixed_cutoff(igpu_batch* batch, double cutoff);

/* Counters of the last J/K or gradient call on the plan. */
int igpu_last_stats(const igpu_plan* plan, igpu_stats* stats);
/* Per-launch records of the last J/K or gradient call (*n = count; at most
 * cap written to out). */
int igpu_last_profile(const igpu_plan* plan, igpu_launch_record* out, size_t cap, size_t* n);
/* Launch-shape autotuner for the J/K launches (no counterpart in the
 * reference, whose CPU path has no launch shapes to tune).  Runs the J/K
 * build of d_dens (device, ndens x nao x nao) at `threshold` and `precision`
 * into scratch outputs it allocates, in two stages, each candidate twice:
 * first per candidate chunk (4, 8, 16, 32 or 64 tasks per team per grab,
 * i.e. quartets per warp per grab), then, with the chosen chunks, per cap on
 * the persistent grid (1, 2, 3 or 4 blocks per SM, or the occupancy limit).
 * It keeps per angular class and precision the candidate of the shortest
 * launch; later J/K calls on the plan use them (16 and the occupancy limit
 * before any tuning).  Results differ only in the order of the atomic
 * additions.  Costs twenty J/K builds. */
int igpu_autotune_jk(igpu_plan* plan, const double* d_dens, int ndens, double threshold, int precision,
                     void* stream);
/* The same two-stage autotuner for the gradient launches: twenty igpu_grad
 * calls on the given (host) term matrices, at threshold and precision, into
 * a scratch output; later gradient calls on the plan use the kept shapes. */
int igpu_autotune_grad(igpu_plan* plan, const igpu_term* coulomb, int ncoul, const igpu_term* exchange,
                       int nexch, double threshold, int precision);

#ifdef __cplusplus
}
#endif

#endif /* INTEGRAL_GPU_H */
