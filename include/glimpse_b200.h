/*
 * glimpse_b200 — C-ABI of the B200 implementation of GLIMPSE2_phase's inner
 * loop: PBWT conditioning-state selection, the haploid Li-Stephens
 * forward-backward (imputation HMM), the 8-hypothesis phasing HMM with Gibbs
 * phase resampling, and genotype-posterior / dosage accumulation.
 *
 * The reference has no FFI for this path; its seams are C++ methods called by
 * the Gibbs driver (phase/src/caller/caller_algorithm.cpp:53-126). Each entry
 * point below names the method(s) it replaces.
 *
 * Conventions
 *  - Every function returns GP_OK (0) or a negative GP_E* status; none exits
 *    or aborts. gp_last_error(ctx) describes the last failure.
 *  - Host buffers are owned by the caller and are only read/written during
 *    the call. Device memory is owned by the context.
 *  - One host thread per context; all work runs on the context's CUDA stream.
 *  - Sites are indexed 0..n_sites-1 in panel order; haplotype bits are 0/1.
 *  - Random numbers come from counter-based streams keyed by
 *    (seed, purpose, iteration, target); see glimpse_b200/csrc/replay_rng.h.
 */
#ifndef GLIMPSE_B200_H
#define GLIMPSE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GP_OK 0
#define GP_E_ARG (-1)      /* invalid argument / size */
#define GP_E_CUDA (-2)     /* CUDA runtime error */
#define GP_E_NOMEM (-3)    /* device or host allocation failed */
#define GP_E_STATE (-4)    /* call out of order (e.g. no targets set) */
#define GP_E_DATA (-5)     /* inconsistent input data (e.g. zero states) */

/* Largest batch per call: targets per context (gp_targets_set; each target
 * has up to 2 haplotypes) and haplotypes or targets per call-level batch
 * (gp_impute_batch, gp_rephase_batch). Batches index the second grid
 * dimension of the kernel launches, whose hardware limit is 65535. */
#define GP_MAX_TARGETS 32767
#define GP_MAX_BATCH 65535

/* Precision modes of the imputation forward-backward (gp_set_precision). */
#define GP_PRECISION_FULL 0       /* every forward row kept in FP32, as the reference keeps them */
#define GP_PRECISION_CKPT_F32 1   /* FP32 checkpoints every 32 sites, FP32 recompute, FP64 log-likelihood */
#define GP_PRECISION_CKPT_BF16 2  /* BF16 checkpoints every 32 sites, FP32 recompute, FP64 log-likelihood */

#define GP_STAGE_INIT 0
#define GP_STAGE_BURN 1
#define GP_STAGE_MAIN 2

typedef struct gp_ctx gp_ctx;

/* Reference panel in the reference's in-memory representation
 * (common/src/containers/ref_haplotype_set.h:60-75, variant.h:33-45). */
typedef struct gp_panel_desc {
  int32_t n_ref_haps;          /* N */
  int32_t n_sites;             /* L */
  const double* cm;            /* [L] genetic position, cM */
  const uint32_t* cref;        /* [L] reference allele count in the panel */
  const uint32_t* calt;        /* [L] alternative allele count in the panel */
  const uint8_t* lq;           /* [L] low-quality site flag (variant::LQ) */
  const uint8_t* flag_common;  /* [L] 1 = common (plain bit matrix), 0 = rare (sparse) */
  const uint8_t* major;        /* [L] major allele (calt > cref) */
  const uint8_t* hvar;         /* HvarRef: n_common rows x ceil(N/8) bytes, MSB first */
  const int64_t* shap_off;     /* ShapRef CSR offsets [N+1] */
  const int32_t* shap_sites;   /* ShapRef CSR values: rare sites carrying the non-major allele */
  /* Optional sparse PBWT (ref_haplotype_set.h:70-71). NULL: built by gp_ctx_create. */
  const uint8_t* ypacked;
  int64_t ypacked_len;
  const int64_t* asmall_off;   /* [n_common_hq + 2] */
  const int32_t* asmall_idx;
} gp_panel_desc;

/* Model and selection parameters (phase/src/caller/caller_parameters.cpp:30-101). */
typedef struct gp_config {
  int32_t ne;                  /* --ne, default 100000 */
  float err_imp;               /* --err-imp, default 1e-12 (clamped to [1e-12, 1e-3]) */
  float err_phase;             /* --err-phase, default 1e-4 */
  float min_gl;                /* --min-gl, default 1e-10 */
  int32_t pbwt_depth;          /* --pbwt-depth, default 12 */
  float pbwt_modulo_cm;        /* --pbwt-modulo-cm, default 0.1 */
  int32_t kinit;               /* --Kinit, default 1000 */
  int32_t kpbwt;               /* --Kpbwt, default 2000 (per-target override in gp_targets_set) */
  uint64_t seed;               /* --seed, default 15052011 */
  int32_t device;              /* CUDA device ordinal */
} gp_config;

/* Fill a config with the reference's defaults. */
void gp_config_defaults(gp_config* cfg);

/* Upload the panel (replaces reading the binary panel in
 * caller_initialise.cpp:93-104 and haplotype_set::allocatePBWT,
 * haplotype_set.cpp:229-315) and create a context. */
int gp_ctx_create(const gp_panel_desc* panel, const gp_config* cfg, gp_ctx** out);
int gp_ctx_destroy(gp_ctx* ctx);
const char* gp_last_error(const gp_ctx* ctx);

/* Targets (genotype_set / genotype objects, genotype.h:81-136).
 * gl: n x L x 3 phred bytes (ploidy+1 used per site), flat: n x L,
 * ploidy: n (1 or 2), kpbwt: n per-target Kpbwt or NULL for cfg->kpbwt. */
int gp_targets_set(gp_ctx* ctx, int32_t n, const uint8_t* gl, const uint8_t* flat, const int32_t* ploidy,
                   const int32_t* kpbwt);

/* Conditioning states always present (--state-list, caller_parameters.cpp:73;
 * haplotype_set::read_list_states, haplotype_set.cpp:835-857). Row h lists
 * reference haplotype ids for target haplotype h (targets in gp_targets_set
 * order, ploidy rows each): ids[offsets[h] .. offsets[h+1]), n_haps = the sum
 * of the ploidies. Every conditioning set of a target then also holds its
 * rows' ids, sorted and without duplicates, except the whole-panel set of
 * Kpbwt >= n_ref_haps (conditioning_set::compactSelection,
 * conditioning_set.cpp:105-121). With lists, cfg->kinit and Kpbwt may be 0:
 * that stage's set is the list alone. gp_targets_set clears the lists;
 * n_haps = 0 clears them too. GP_E_ARG for a row count other than the
 * targets' haplotypes, an empty row (the reference's "List of states for
 * haplotype h is empty") or an id outside [0, n_ref_haps); at selection, for a
 * stage whose K plus the longest list exceeds 2048 states. */
int gp_state_lists_set(gp_ctx* ctx, int32_t n_haps, const int64_t* offsets, const int32_t* ids);

/* Target GL input (genotype_reader::readTargetGenotypes, genotype_reader.cpp:427-500):
 * the FORMAT/PL (int32) or FORMAT/GL (float) values of n targets at L sites,
 * as htslib's bcf_get_format_int32 / bcf_get_format_float return them per
 * site, packed site after site: value c of target i at site l is
 * src[(l * n + i) * P + c], P = max(ploidy) + 1. site_nval[l] is the value
 * count htslib returned for site l (NULL: n * P at every site); a site whose
 * count / n differs from P is skipped, as the reference skips it. Writes gl
 * (n x L x 3 phred bytes: PL, or lroundf(-10 GL), clamped to 255) and flat
 * (n x L), the layout gp_targets_set takes. Absent values (missing or vector
 * end) leave a target's site at phred 0 and flat. A negative PL or a positive
 * GL returns GP_E_DATA naming the first such (site, target). */
int gp_gl_from_pl(gp_ctx* ctx, int32_t n, int32_t L, const int32_t* pl, const int32_t* site_nval,
                  const int32_t* ploidy, uint8_t* gl, uint8_t* flat);
int gp_gl_from_float(gp_ctx* ctx, int32_t n, int32_t L, const float* glf, const int32_t* site_nval,
                     const int32_t* ploidy, uint8_t* gl, uint8_t* flat);

/* One Gibbs iteration over all targets (caller::phase_iteration,
 * caller_algorithm.cpp:86-126, with phase_individual :53-84 for every target):
 * selection, haplotype likelihoods, two imputation passes with sampling,
 * phasing, and in the main stage the genotype-posterior accumulation.
 * iteration keys the random streams (0 = init, then 1, 2, ...). */
int gp_iteration(gp_ctx* ctx, int32_t stage, int32_t iteration);

/* Whole run: 1 init + burnin + main iterations, then finalisation
 * (caller::phase_loop, caller_algorithm.cpp:223-243). */
int gp_run(gp_ctx* ctx, int32_t burnin, int32_t main);

/* Current haplotypes (checkpoint/resume stays with the caller,
 * caller_algorithm.cpp:136-221). h0/h1: n x L bytes. */
int gp_haps_get(gp_ctx* ctx, uint8_t* h0, uint8_t* h1);
int gp_haps_set(gp_ctx* ctx, const uint8_t* h0, const uint8_t* h1);

/* Per-site haplotype posteriors of the last iteration for one target
 * (HP0/HP1 of phase_individual): hp0/hp1: 2 x L floats. */
int gp_posteriors_get(gp_ctx* ctx, int32_t target, float* hp0, float* hp1);

/* Conditioning states of the last iteration for one target
 * (conditioning_set::idxHaps_ref, conditioning_set.h:62). Returns the count
 * through n_out; states must hold at least n_ref_haps entries. */
int gp_states_get(gp_ctx* ctx, int32_t target, uint32_t* states, int32_t* n_out);

/* Finalised genotype posteriors and dosages (genotype::sortAndNormAndInferGenotype,
 * genotype.cpp:211-244, and the DS/GP fields of genotype_writer.cpp:98-160):
 * all arrays n x L. gp0/gp1 as stored (GP of genotypes 0 and 1), ds the dosage
 * gp1 + 2*gp2 rounded to 1e-3, gt0/gt1 the called alleles (hds-phased hets). */
int gp_finalize(gp_ctx* ctx);
int gp_gp_get(gp_ctx* ctx, float* gp0, float* gp1, float* ds, uint8_t* gt0, uint8_t* gt1);

/* Parity hook: the genotype-posterior accumulators of one target as they
 * stand (genotype::stored_data, genotype.h:38-78, before or after gp_finalize),
 * dense over the L sites: gp0/gp1 the stored sums (normalised once finalised),
 * flags bit 0 = an entry exists for the site (created when p0 / sum < 0.99999,
 * genotype.cpp:127-209), bit 1 = hds. Sites without an entry read gp0 = gp1 = 0. */
int gp_gp_accum_get(gp_ctx* ctx, int32_t target, float* gp0, float* gp1, uint8_t* flags);

/* The record fields genotype_writer::writeGenotypes computes beyond GT and DS
 * (genotype_writer.cpp:110-190), after gp_finalize: gp (n x L x 3) the FORMAT/GP
 * values as written (floored to 1e-3, then raised by 1e-3 in the writer's order
 * until they sum to 0.9999; a haploid target's third value is htslib's
 * vector-end marker), and per site raf (calt / (calt + cref)), af (sum of DS over
 * target haplotypes) and info (the INFO score; 1 unless every target is
 * diploid and 0 < af < 1; the writer omits it for mixed ploidy). */
int gp_output_records(gp_ctx* ctx, float* gp, float* raf, float* af, float* info);

/* ---- Ligation of consecutive chunks (GLIMPSE2_ligate) ---- */

/* Phase-flip counting over the overlap of two consecutive chunks
 * (ligater::update_distances and the decision in ligater::scan_overlap,
 * ligater_algorithm.cpp:108-127,183-205). gta / gtb: htslib GT values (2 int32
 * per sample) of the m bi-allelic sites present in both chunks, site after site
 * (m x n x 2). swap_prev: the swap decided for the first chunk. Writes swap_next
 * (nmatch < nmism), the per-sample counts and the entropy phase quality.
 * m = 0 returns GP_E_DATA ("Overlap is empty"). */
int gp_ligate_overlap(gp_ctx* ctx, int32_t n, int32_t m, const int32_t* gta, const int32_t* gtb,
                      const uint8_t* swap_prev, uint8_t* swap_next, int32_t* nmatch, int32_t* nmism, float* phaseq);

/* ligater::phase_update (ligater_algorithm.cpp:90-106) on m records of a chunk,
 * in place: for every sample with swap[i], a phased diploid GT becomes
 * (allele 2 == 1, allele 1 == 1), phased. gt: m x n x 2 htslib GT values. */
int gp_ligate_swap(gp_ctx* ctx, int32_t n, int32_t m, int32_t* gt, const uint8_t* swap);

/* ---- Call-level entry points (one reference method, batched) ---- */

/* imputation_hmm::computePosteriors(HL, flat, HP) (imputation_hmm.h:59)
 * for n independent haplotypes, each with an explicit conditioning set given
 * as sorted reference-haplotype ids (states_off[n+1], states). hl, hp: n x 2L;
 * flat: n x L. The conditioning set is built as
 * conditioning_set::compactSelection builds it (conditioning_set.cpp:123-196). */
int gp_impute_batch(gp_ctx* ctx, int32_t n, const int64_t* states_off, const uint32_t* states, const float* hl,
                    const uint8_t* flat, float* hp);

/* No counterpart in the reference. The same computation as gp_impute_batch
 * with n = 1 (k sorted state ids; hl, hp: 2L floats; flat: L bytes), for
 * callers that must not allocate device memory during the call: all scratch
 * lives in one fixed 64 MiB region per device inside the library. The per-site
 * buffers take about 51 x n_sites bytes plus n_sites / 32 x k x 4; the
 * forward-backward store takes (polymorphic sites of the conditioning set) x
 * k x 4 bytes from the rest. A call that does not fit returns GP_E_ARG before
 * the HMM runs. The first call on a device looks the region up and should come
 * before any stream capture. Overlapping calls on one device race. */
int gp_impute_one_static(gp_ctx* ctx, int32_t k, const uint32_t* states, const float* hl, const uint8_t* flat,
                         float* hp);

/* Precision of the imputation forward-backward for every later call (no
 * counterpart in the reference, which keeps every forward row,
 * imputation_hmm.cpp:53-59). GP_PRECISION_FULL (the default) keeps all rows in
 * FP32. The checkpointed modes keep the forward row after every 32nd
 * polymorphic site only (FP32 or BF16; about 1/32 or 1/64 of the memory),
 * recompute each block's rows in FP32 during the backward pass, and accumulate
 * the chunk log-likelihood sum_l log AlphaSum_l in FP64 (gp_loglik_get). With
 * FP32 checkpoints the posteriors are those of the same recursion without
 * checkpoints; BF16 checkpoints trade a small posterior error for memory. */
int gp_set_precision(gp_ctx* ctx, int32_t mode);

/* The FP64 chunk log-likelihood of each haplotype of the last imputation call
 * made in a checkpointed mode (n entries, in the call's order; for a Gibbs
 * iteration: the targets' second haplotypes, or first for haploid targets). */
int gp_loglik_get(gp_ctx* ctx, int32_t n, double* out);

/* phasing_hmm::rephaseHaplotypes(H0, H1, flat) (phasing_hmm.h:136) for n
 * diploid targets with explicit conditioning sets; h0/h1 updated in place
 * (n x L). Target t draws from stream (RNG_PHASE, iteration, target_ids[t]). */
int gp_rephase_batch(gp_ctx* ctx, int32_t n, const int64_t* states_off, const uint32_t* states, uint8_t* h0,
                     uint8_t* h1, const uint8_t* flat, int32_t iteration, const int32_t* target_ids);

/* haplotype_set::matchHapsFromCompressedPBWTSmall (haplotype_set.cpp:317-394)
 * from the current target haplotypes, followed by the state union of
 * conditioning_set::compactSelection (conditioning_set.cpp:96-104). */
int gp_select(gp_ctx* ctx, int32_t stage, int32_t iteration);

/* pbwt_states of the last selection for one target, level by level
 * (haplotype_set.h:95): fills counts[pbwt_depth] and states (concatenated). */
int gp_pbwt_states_get(gp_ctx* ctx, int32_t target, int32_t* counts, int32_t* states, int32_t cap);

/* Sparse PBWT of the panel (ref_haplotype_set::build_sparsePBWT,
 * ref_haplotype_set.cpp:47-103): returns lengths, copies when buffers are given. */
int gp_sparse_pbwt_get(gp_ctx* ctx, uint8_t* ypacked, int64_t* ypacked_len, int64_t* asmall_off,
                       int32_t* asmall_idx, int64_t* asmall_len);

/* The same sparse PBWT built from a panel descriptor on the host, without a
 * context or a GPU (offline panel preparation, as GLIMPSE2_split_reference
 * does through ref_haplotype_set::build_sparsePBWT). Call once with NULL
 * buffers to get the lengths; asmall_off has n_common_hq + 2 entries. */
int gp_build_sparse_pbwt(const gp_panel_desc* panel, uint8_t* ypacked, int64_t* ypacked_len, int64_t* asmall_off,
                         int32_t* asmall_idx, int64_t* asmall_len);

/* ---- Learned state-selection proposal: the scoring network ----
 * No counterpart in the reference, which selects conditioning states by PBWT
 * alone (haplotype_set.cpp:682-728, conditioning_set.cpp:96-104). An MLP
 * scores candidate reference haplotypes from 48 features per candidate:
 * 48 -> 256 -> 256 -> 1 with ReLU, BF16 weights and activations, FP32
 * accumulation, forward and backward on the tensor cores. Parameters are one
 * packed FP32 vector of gp_mlp_param_count() values: W1 [256][64] (row = hidden
 * unit; columns 48..63 are padding and must be zero), b1 [256], W2 [256][256]
 * (row = output unit), b2 [256], w3 [256], b3 [1]. */
int32_t gp_mlp_param_count(void);
/* He-uniform weights from a seed, zero biases; resets the optimiser. */
int gp_mlp_init(gp_ctx* ctx, uint64_t seed);
int gp_mlp_set_params(gp_ctx* ctx, const float* params);
int gp_mlp_get_params(gp_ctx* ctx, float* params);
/* Scores of n feature rows x (n x 48 FP32, rounded to BF16 on the device);
 * h1, h2 (n x 256, optional) receive the BF16 hidden activations. */
int gp_mlp_forward(gp_ctx* ctx, int32_t n, const float* x, float* score, float* h1, float* h2);
/* One training step on n rows: loss = sum_i wt_i BCE(sigmoid(score_i), y_i) / n
 * (wt NULL: 1), gradients by the backward kernels, then one Adam step with
 * learning rate lr (lr = 0: no update). loss and grad (gp_mlp_param_count()
 * values, before the update) are optional outputs. */
int gp_mlp_train_step(gp_ctx* ctx, int32_t n, const float* x, const float* y, const float* wt, float lr, float* loss,
                      float* grad);

/* ---- Learned state-selection proposal ----
 * No counterpart in the reference. With it enabled, burn-in and main
 * iterations select each target's conditioning states in place of the union of
 * conditioning_set::compactSelection (conditioning_set.cpp:96-104): the PBWT
 * selection (haplotype_set.cpp:317-728) runs with kcand states per target to
 * give candidates; every (target, window of 256 common sites, candidate) gets
 * 48 features (the candidate's PBWT level and rank in the PBWT union order,
 * matches with the target's two current haplotypes over the window and its
 * neighbours, match runs through the window, agreement with confident
 * genotype-likelihood calls, densities); the network scores them;
 * per window the top 32 candidates are ranked, and the conditioning set is the
 * union in rank order cut at the target's Kpbwt (gp_targets_set). The init
 * stage is unchanged. Disabled (the default), selection is the plain PBWT path.
 * Enabling needs network parameters (gp_mlp_init, gp_mlp_set_params or
 * gp_learned_train); kcand is at most 2048. */
int gp_learned_enable(gp_ctx* ctx, int32_t enable, int32_t kcand);

/* Size of the learned proposal's conditioning sets. kmin = 0 (the default):
 * each target's Kpbwt. kmin > 0: the candidates that some window scores at
 * probability min_prob or more (the network's estimate of y, see
 * gp_learned_train), at least kmin, at most the target's Kpbwt; the size
 * then follows how many haplotypes the target's windows need. */
int gp_learned_size(gp_ctx* ctx, float min_prob, int32_t kmin);

/* Windows of the learned proposal: runs of 256 consecutive common sites; a
 * rare site belongs to the window of the last common site before it. */
int32_t gp_learned_windows(gp_ctx* ctx);

/* Per-window state posteriors (the learned proposal's training labels) for n
 * haplotypes with explicit conditioning sets, as gp_impute_batch takes them:
 * the HMM of imputation_hmm (imputation_hmm.cpp:80-353) over the set, with
 * per-site normalisation; for haplotype i, window w and state j of its set,
 * mass[nwin * states_off[i] + w * K_i + j] = sum over the window's polymorphic
 * sites of alpha(j) beta(j) / sum_j' alpha(j') beta(j'); nsites (n x nwin)
 * counts those sites. nwin = gp_learned_windows(ctx). */
int gp_state_posteriors(gp_ctx* ctx, int32_t n, const int64_t* states_off, const uint32_t* states, const float* hl,
                        const uint8_t* flat, float* mass, int32_t* nsites);

/* Train the network on the context's current targets and haplotypes (run a few
 * plain iterations first): candidates from the PBWT selection at kcand; labels
 * from the HMM over all candidates of each target, per window the larger of the
 * two haplotypes' posterior share q of a candidate, y = min(1, kpos q), weight
 * 1 + 10 y; then `steps` Adam steps (learning rate lr) on batches of `batch`
 * rows (a multiple of 128) drawn without replacement, reshuffled each pass.
 * losses (optional, steps values) receives each step's loss. Initialises the
 * network from seed when it has no parameters. */
int gp_learned_train(gp_ctx* ctx, int32_t kcand, float kpos, int32_t steps, int32_t batch, float lr, uint64_t seed,
                     float* losses);

/* Launch-shape autotuner (no counterpart in the reference). Two shapes are
 * picked per context by timing every candidate on the first batch large
 * enough to tell them apart (16 haplotypes for the imputation chains, 32 target
 * haplotypes for the PBWT sweep): chains per CTA of the imputation
 * forward-backward (1, 2 or 4: how many sequential chains share an SM's
 * shared memory and schedulers) and target haplotypes per warp of the PBWT
 * sweep (1, 2, 4 or 8: lockstep lanes against divergence). Results do not
 * depend on either. gp_tuning_set fixes them (0: tune again on next use);
 * gp_tuning_get reports the shapes in use (0: not tuned yet) and, in ms[7],
 * the measured times (phase-1 chains for 1, 2, 4 chains per CTA, then the sweep
 * for 1, 2, 4, 8 haplotypes per warp; -1 where a shape did not fit, 0 where
 * not measured). A third choice, set by the caller and not timed (the two
 * measured alike), is the placement of the phasing CTAs when a batch has one
 * to two entries per SM (phase_placement 1, the default: entries in
 * decreasing order of work; 2: the heaviest alone on an SM and the others
 * paired heaviest with lightest). ms holds 9 floats; the last two are 0. */
int gp_tuning_set(gp_ctx* ctx, int32_t chains_per_cta, int32_t sweep_haps_per_warp, int32_t phase_placement);
int gp_tuning_get(gp_ctx* ctx, int32_t* chains_per_cta, int32_t* sweep_haps_per_warp, int32_t* phase_placement,
                  float* ms);

/* Timing of the last gp_iteration by stage, in milliseconds (device events). */
int gp_stage_times(gp_ctx* ctx, float* ms, int32_t n);

/* Counters accumulated since the last gp_profile_reset: device time of the
 * imputation forward-backward and phasing kernels (CUDA events around each
 * launch on the context stream), their algorithmic work, and the number of
 * kernels this library launched. */
typedef struct gp_profile {
  double impute_ms, impute_cells, impute_bytes;  /* cells = sum over launches of poly sites x states */
  double phase_ms, phase_cells;                  /* cells = VAR sites x states x 8 hypotheses, both passes */
  double select_ms;
  int64_t impute_launches, phase_launches, kernel_launches;
  double mlp_ms, mlp_rows;                       /* the learned proposal's fused forward (k_mlp_fwd) */
  int64_t mlp_launches;
} gp_profile;
int gp_profile_get(gp_ctx* ctx, gp_profile* out);
int gp_profile_reset(gp_ctx* ctx);

/* The CUDA stream the context runs on (a cudaStream_t), for callers that time
 * or order their own work around the library's. */
void* gp_stream(gp_ctx* ctx);

/* Reset all targets to the state gp_targets_set leaves them in (haplotypes 0,
 * no stored posteriors) without re-reading any host buffer. */
int gp_targets_reset(gp_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* GLIMPSE_B200_H */
