/*
 * fmmcuda.h: C ABI of the B200 fast-multipole Biot-Savart solver (libfmmcuda.so).
 *
 * The reference (iamwhoamianamy/bachelors) exposes its GPU code through the C++-ABI
 * "kernel_callers" seam (FMMCUDADLL/kernel_callers.hpp:5-10, kernels::addVectors, and the
 * live twin FMM/FMMGPU/translation_algorithms.hpp:8-61, kernels::translateAll*) and its
 * solver through C++ classes (FMM/FMMGPU/multipole_solver.hpp:12-48,
 * FMM/FMMGPU/fast_multipole_solver.hpp:13-49). This header replaces both with plain
 * extern "C" entry points: pointers, sizes and integer status codes, no C++ or torch types.
 *
 * Physics (FMM/FMMGPU/integration.cpp:101-161, fast_multipole_solver.cpp:195-231):
 *   B(x) = MU0 / (4 PI) * current * sum_q w_q J_q x (x - q) / |x - q|^3
 *   A(x) = 1 / (4 PI) * current * sum_q w_q J_q / |x - q|
 * with the reference's literals PI = 3.14159265359 and MU0 = 1.2566370614e-6
 * (FMM/FMMGPU/math.hpp:12-13). Coincident (target, source) pairs are skipped.
 *
 * Errors: every call returns an fmm_status; fmm_last_error_string() describes the last
 * failure on the calling thread. Nothing here exits the process (the reference prints and
 * calls exit(0), FMM/FMMGPU/cuda_helper.cpp:9-31).
 *
 * Threading: a plan is used by one host thread at a time; distinct plans are independent.
 * Work is issued on the stream passed to each call (NULL = the legacy default stream).
 */
#ifndef FMMCUDA_H
#define FMMCUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum fmm_status {
   FMM_OK = 0,
   FMM_E_INVALID = 1, /* bad argument or call order */
   FMM_E_OOM = 2,     /* device allocation failed */
   FMM_E_CUDA = 3,    /* a CUDA runtime or launch error */
   FMM_E_TIMEOUT = 4, /* a bounded device wait ran out */
   FMM_E_LIMIT = 5    /* a structural limit was exceeded (tree depth, list capacity) */
} fmm_status;

/* Arithmetic of the whole pipeline. FP64 also builds every operator table in FP64. */
typedef enum fmm_precision { FMM_FP32 = 0, FMM_FP64 = 1 } fmm_precision;

/* How the M2L contraction is computed (FP32 plans only; FP64 plans always use FMM_M2L_SIMT).
 *   SIMT    FP32 (or FP64) FMA on the CUDA cores.
 *   BF16X3  tcgen05 tensor cores, operands split x = hi + lo in bf16, hi*hi + hi*lo + lo*hi,
 *           FP32 accumulation in tensor memory (about 16 bits per product).
 *   TF32    tcgen05 tensor cores, one TF32 pass, FP32 accumulation.
 *   BF16X6  tcgen05 tensor cores, operands split x = hi + mid + lo in bf16 and the six products
 *           down to 2^-16 relative kept (about FP32 accuracy). */
typedef enum fmm_m2l_mode {
   FMM_M2L_SIMT = 0,
   FMM_M2L_BF16X3 = 1,
   FMM_M2L_TF32 = 2,
   FMM_M2L_BF16X6 = 3
} fmm_m2l_mode;

typedef struct fmm_config {
   int order;          /* expansion order p, 1..16 ((p+1)^2 harmonics) */
   int leaf_capacity;  /* a box splits when it holds more than this many sources ... */
   int target_leaf_capacity; /* ... or more than this many targets (<= 0: leaf_capacity) */
   int precision;      /* fmm_precision */
   int m2l_mode;       /* fmm_m2l_mode */
   int m2l_truncate;   /* 0: full M2L operator (l + lambda <= 2p); 1: the reference's l + lambda <= p
                          (FMM/FMMGPU/multipole_translator.cpp:165) */
   int device;         /* CUDA device ordinal */
   double root_center[3];
   double root_half_width; /* <= 0: the cube around the bounding box of sources and targets */
   int m2l_tc_degree_cutoff; /* tensor-core M2L modes: translation terms with l + lambda above this are
                                dropped (they decay like (box size / distance)^(l + lambda)); 0: p + 8,
                                which keeps the FP64 truncation error near that of the full operator
                                (about 1e-7 relative at p = 16); < 0: the full operator (l + lambda <= 2p);
                                values below p are raised to p */
} fmm_config;

typedef struct fmm_plan fmm_plan;

/* Phase timings (milliseconds, CUDA events on the plan's stream) and tree statistics of
 * the last solve. */
typedef struct fmm_stats {
   double ms_tree, ms_upward, ms_m2l, ms_downward, ms_near, ms_total;
   int64_t nodes, leaves, levels, v_pairs, p2p_pairs, p2p_interactions;
   /* boxes, leaf boxes, levels, M2L (V-list) box pairs, direct (leaf, source box) pairs, and the direct
      (target, source) point pairs the near field evaluates */
   int64_t n_sources, n_targets;
   double ms_adjoint; /* the last fmm_adjoint call */
   int64_t coils;     /* independent problems in the plan (1 unless batched) */
   int64_t m2l_tiles, m2l_tile_offsets; /* tensor-core M2L: 42-box tiles and (tile, offset) steps;
                                           the row fill is 3 v_pairs / (128 m2l_tile_offsets) */
} fmm_stats;

void fmm_default_config(fmm_config* cfg);

/* Replaces MultipoleSolver / FastMultipoleSolver construction
 * (FMM/FMMGPU/multipole_solver.cpp:20-36, fast_multipole_solver.cpp:12-23). */
fmm_status fmm_plan_create(const fmm_config* cfg, fmm_plan** plan);
fmm_status fmm_plan_destroy(fmm_plan* plan);

/* Sources: xyz[3n], weights w[n], current directions J[3n] (J == NULL: the reference's
 * azimuthal direction perp(q)/|perp(q)|, FMM/FMMGPU/integration.cpp:155). Element type is
 * float for FP32 plans and double for FP64 plans. on_device != 0: the pointers are device
 * memory on the plan's device; otherwise host memory (copied on `stream`). The data is
 * copied; the caller's buffers may be released after the call returns. */
fmm_status fmm_set_sources(fmm_plan* plan, const void* xyz, const void* w, const void* J, int64_t n,
                           int on_device, void* stream);
/* fmm_set_sources for page-locked host buffers (cudaHostAlloc / cudaHostRegister; anything else is
 * FMM_E_INVALID), without waiting for the copies: the points, then the weights and directions, cross the
 * bus on a copy stream of the plan, after the work queued on `stream` so far. The next tree build
 * (fmm_build_tree / fmm_solve) starts once the points are in and takes the strengths at its end, so
 * their copy runs under the build; every other call that reads the sources waits for the copies on
 * its stream. The caller keeps the buffers alive and unchanged until the next fmm_solve (or
 * fmm_build_tree) on this plan has returned. No counterpart in the reference, whose sources live in
 * host memory. */
fmm_status fmm_set_sources_async(fmm_plan* plan, const void* xyz, const void* w, const void* J, int64_t n,
                                 void* stream);
/* BEM sources (the reference's Problem::BEM, FMM/FMMGPU/multipole_solver_enums.hpp:26-30, BEMQuadrature
 * bem_quadrature.hpp): points xyz[3n], weights w[n], field values B[3n] and surface normals normal[3n]. The
 * plan then computes the reference's BEM integral (math::calcBEMIntegral, integration.cpp:191-215)
 *   F(x) = 1/(4 PI) sum_q w_q [(B_q . n_q) d + d x (B_q x n_q)] / |d|^3,  d = q - x,
 * by fmm_solve / fmm_evaluate (FastMultipoleSolver::calcBEM, fast_multipole_solver.cpp:233-250; the
 * multipoles are those of math::calcBEMIntegralContribution, integration.cpp:295-353, from the analytic
 * gradient of the regular harmonics; close boxes are summed directly) and fmm_direct, always with want = 2,
 * the result in out_A and no current factor, as there; fmm_treecode (want = 2) scales it by `current` as
 * MultipoleSolver::calcA does. Not available with fmm_adjoint, fmm_update_sources or batches.
 * fmm_set_sources returns the plan to the Biot-Savart problem. */
fmm_status fmm_set_bem_sources(fmm_plan* plan, const void* xyz, const void* w, const void* B, const void* normal,
                               int64_t n, int on_device, void* stream);

/* Targets xyz[3m] (FastMultipoleSolver's `points`, fast_multipole_solver.hpp:16). */
fmm_status fmm_set_targets(fmm_plan* plan, const void* xyz, int64_t m, int on_device, void* stream);
/* Targets = the current source points, in source input order (no counterpart in the reference, whose
 * FastMultipoleSolver always takes its own `points`): a device-side copy on `stream`, so a caller
 * evaluating B at its own quadrature points moves them to the GPU once. A single-coil plan's tree build
 * then reuses the sources' sorted order for the targets (one sort instead of two). The targets stay
 * these points until the next fmm_set_targets or fmm_set_targets_to_sources, also when new sources
 * are set. */
fmm_status fmm_set_targets_to_sources(fmm_plan* plan, void* stream);

/* The reference's phases, for drop-in use of its call sequence
 * (FMM/FMMGPU/main.cpp:568-572):
 *   fmm_build_tree          <- initTrees (multipole_solver.cpp:656-675, fast_multipole_solver.cpp:43-60)
 *   fmm_upward              <- calcMultipoleExpansionsAtLeaves + calclMultipoleExpansions
 *   fmm_downward            <- calcLocalMultipoleExpansions (M2L + L2L)
 *   fmm_evaluate            <- calcB(current) / calcA(current) (L2P + direct near field)
 * Each runs on `stream` and requires the previous phase. */
fmm_status fmm_build_tree(fmm_plan* plan, void* stream);
fmm_status fmm_upward(fmm_plan* plan, void* stream);
fmm_status fmm_downward(fmm_plan* plan, void* stream);
/* want: 1 = B, 2 = A, 3 = both. out_B / out_A hold 3m values in target input order, in the
 * plan's element type, on the device (on_device != 0) or host. */
fmm_status fmm_evaluate(fmm_plan* plan, double current, int want, void* out_B, void* out_A, int on_device,
                        void* stream);

/* All phases in order. */
fmm_status fmm_solve(fmm_plan* plan, double current, int want, void* out_B, void* out_A, int on_device,
                     void* stream);

/* Treecode point queries (MultipoleSolver::calcA / calcB(current, point), FMM/FMMGPU/multipole_solver.cpp:686-700,
 * with QuadratureOctreeNode::calcA / calcRot, quadrature_octree.cpp:171-258): B and/or A at pts[3m] from the
 * plan's source tree and multipoles (call fmm_build_tree and fmm_upward first; the plan's own targets play no
 * part, and a plan without targets has the reference's source-only tree). For each point the tree is walked
 * from the root: a box of half-diagonal r at distance d from the point contributes its multipole when
 * 4 r^2 < d^2, otherwise its children do; a leaf that fails the test is summed directly, and B comes from the
 * analytic gradient of the irregular harmonics. Flags reproduce the reference's choices instead:
 * FMM_TREECODE_REFERENCE_NEAR drops such leaves (they contribute nothing there), FMM_TREECODE_FD_CURL takes B
 * by central differences of A with step 1e-3. The reference's tree uses root centre 0 and half-width 3 and
 * splits a box holding `cap` points: configure root_center / root_half_width and leaf_capacity = cap - 1.
 * Outputs in point input order, the plan's element type; not available on a batched plan. */
#define FMM_TREECODE_REFERENCE_NEAR 1
#define FMM_TREECODE_FD_CURL 2
fmm_status fmm_treecode(fmm_plan* plan, double current, int want, const void* pts, int64_t m, void* out_B, void* out_A,
                        int flags, int on_device, void* stream);

/* Direct O(N M) sums on the device in the plan's precision, over the plan's current
 * sources and targets (math::calcBioSavartLaplace, FMM/FMMGPU/integration.cpp:101-111). */
fmm_status fmm_direct(fmm_plan* plan, double current, int want, void* out_B, void* out_A, int on_device,
                      void* stream);

/* FP64 direct B on the device for an explicit target subset (accuracy checks): tgt[3k]
 * host doubles, out_B[3k] host doubles. Uses the plan's sources. */
fmm_status fmm_direct_fp64_subset(fmm_plan* plan, double current, const double* tgt, int64_t k, double* out_B);

/* Adjoint FMM (no counterpart in the reference, which has no gradients). Given dLoss/dB at the
 * plan's targets, g[3m], returns dLoss/dJ[3n] and dLoss/d(source positions)[3n] (either output may
 * be NULL) for B as computed by fmm_solve with the same `current`:
 *   dLoss/dJ_q = MU0 I/(4 PI) w_q sum_t g_t x (q - x_t)/|q - x_t|^3
 *   dLoss/dq   = MU0 I/(4 PI) w_q grad_q (J_q . C(q)),  C(q) = sum_t g_t x (q - x_t)/|q - x_t|^3
 * (plus the derivative of the azimuthal direction when J was NULL). It runs one FMM on the
 * swapped point sets (targets as sources of strength g) with first and second derivatives of the
 * local expansions. Weights are constants. Element type and on_device as in fmm_evaluate. */
fmm_status fmm_adjoint(fmm_plan* plan, double current, const void* dL_dB, void* dL_dJ, void* dL_dx, int on_device,
                       void* stream);

/* The same gradients as fmm_adjoint by direct O(N M) summation (FP64 accumulation, results in the
 * plan's element type), for checking the adjoint FMM and for small problems. Needs only sources and
 * targets (no tree); respects the coils of a batched plan. */
fmm_status fmm_adjoint_direct(fmm_plan* plan, double current, const void* dL_dB, void* dL_dJ, void* dL_dx,
                              int on_device, void* stream);

/* Batching (no counterpart in the reference, which solves one coil per solver object): many
 * independent problems ("coils") in one plan. Coil c owns the sources [src_offsets[c], src_offsets[c+1])
 * and the targets [tgt_offsets[c], tgt_offsets[c+1]) of the arrays given to fmm_set_sources /
 * fmm_set_targets (so each coil's points are contiguous there); its sources act only on its targets.
 * Each coil gets its own root cube (around its own points; root_center / root_half_width are
 * ignored) and every phase processes all coils in the same launches, level by level. Offsets are
 * host arrays of ncoils + 1 entries from 0 to n (resp. m); call after fmm_set_sources and
 * fmm_set_targets. ncoils = 0 returns the plan to a single problem. fmm_direct, fmm_adjoint and the
 * graph calls respect the coils; fmm_direct_fp64_subset is not available on a batched plan. */
#define FMM_MAX_COILS 65536
fmm_status fmm_batch_set_coils(fmm_plan* plan, int64_t ncoils, const int64_t* src_offsets, const int64_t* tgt_offsets);

/* Sharding a batch of coils over ranks (no counterpart in the reference, which runs on one device): assigns
 * each of the ncoils coils (offsets as for fmm_batch_set_coils) to one of nparts parts so that the parts'
 * work (sources + targets of their coils) is balanced: coils by decreasing work, each to the least-loaded
 * part (ties to the lower part). Host only and deterministic, so every rank computes the same assignment;
 * each rank then builds a batched plan of its part's coils. No data path crosses ranks except the
 * gathering of the results, which is the caller's (bachelors_b200/sharding.py does it with
 * torch.distributed). part[c] receives the part of coil c. */
fmm_status fmm_batch_partition(int64_t ncoils, const int64_t* src_offsets, const int64_t* tgt_offsets, int nparts,
                               int* part);

/* Tile choices of the kernels (no counterpart in the reference, whose kernels have fixed shapes).
 * Every choice computes the same result up to rounding; they differ in speed with the order, the
 * leaf sizes and the point distribution. */
typedef struct fmm_tuning {
   int m2l_k_chunk;  /* tensor-core M2L: K chunk width, 64 (two 108 KB stages at p = 16) or 32 (four) */
   int near_tile;    /* near field: source points per shared-memory tile, 128 or 256 */
   int p2m_chunk;    /* P2M: 0 = one warp per leaf (lanes own harmonic orders); 16 or 32 = one block
                        per leaf, that many recurrence steps reduced per shared-memory tile */
   double ms_upward, ms_downward, ms_near; /* fmm_autotune: the chosen variants' times */
} fmm_tuning;

/* The project's autotuner: times every variant of each choice on the plan's current data (call it
 * after an fmm_solve, which builds the tree), keeps the fastest and records it for plans created
 * later in this process with the same device, order, leaf capacities, precision and M2L mode (they
 * start with it). The plan's expansions stay valid; `out` may be NULL. Synchronises `stream`. */
fmm_status fmm_autotune(fmm_plan* plan, fmm_tuning* out, void* stream);
fmm_status fmm_get_tuning(const fmm_plan* plan, fmm_tuning* out);
fmm_status fmm_set_tuning(fmm_plan* plan, const fmm_tuning* tuning);

/* New weights w[n] and currents J[3n] for the same source positions (J must be NULL exactly when
 * the sources were set without J). Keeps the tree; the next solve or graph launch uses them. */
fmm_status fmm_update_sources(fmm_plan* plan, const void* w, const void* J, int on_device, void* stream);

/* CUDA graph of one solve on the current tree: P2M, M2M, M2L, L2L and L2P + near field, captured
 * once (after an fmm_solve, which builds the tree, operators and buffers) and replayed by
 * fmm_graph_launch, typically after fmm_update_sources. want: 1 = B, 2 = A, 3 = both. The graph is
 * dropped when sources, targets or the tree change. fmm_graph_launch scales by `current` and writes
 * out_B / out_A (device or host as on_device says). */
fmm_status fmm_graph_capture(fmm_plan* plan, int want, void* stream);
fmm_status fmm_graph_launch(fmm_plan* plan, double current, void* out_B, void* out_A, int on_device, void* stream);

/* Limit of one bounded wait in the tensor-core pipelines (no counterpart in the reference, whose
 * kernels have no device-side waits). Every producer/consumer wait of the tcgen05 M2L, M2M and L2L
 * gives up after this many seconds (default 2; range (0, 60]); the call that ran the pipeline then
 * returns FMM_E_TIMEOUT, the plan stays usable, and the next call recomputes what it needs. The
 * device error word is read once at the end of fmm_solve (and of fmm_upward, fmm_downward,
 * fmm_adjoint, fmm_autotune, and fmm_graph_launch with host outputs), not after every launch.
 * A graph captured earlier is dropped (it holds the old limit). */
fmm_status fmm_set_wait_limit(fmm_plan* plan, double seconds);

fmm_status fmm_get_stats(const fmm_plan* plan, fmm_stats* stats);

/* Operator tables, for verification. kind 0 = M2M (index = child octant 0..7), 1 = L2L
 * (octant 0..7), 2 = M2L (index = offset (ox+3) + 7 (oy+3) + 49 (oz+3), |o|_inf in 2..3).
 * out[(p+1)^2 * (p+1)^2], row-major [output coefficient][input coefficient], FP64, in the
 * box-size-scaled basis the pipeline uses. */
fmm_status fmm_get_operator(fmm_plan* plan, int kind, int index, double* out);

/* No counterpart in the reference. The direct FP32 sum of fmm_direct (B only, coincident pairs
 * skipped, J == NULL: azimuthal direction) for callers that cannot let a library allocate device
 * memory: their GPU memory belongs to another allocator, or their host loop cannot afford a
 * cudaMalloc that may synchronise the device or fail. Inputs xyz[3n], w[n], J[3n] (or NULL) and
 * tgt[3m] and the output out_B[3m] are device pointers on the current device; work is queued on
 * `stream` and the call does not wait for it. The only scratch, the packed sources, lives in a
 * fixed 8 MiB device array inside the library, present on every GPU that loads it until the
 * process exits: n is limited to 262,144 sources (FMM_E_LIMIT beyond). The first call on a device
 * loads the array onto it (CUDA loads a library's device module lazily) and looks up its address:
 * that call may allocate the array's 8 MiB and synchronise, and fails with FMM_E_CUDA when another
 * allocator has already reserved all of the device's memory, so make it once per device before such
 * an allocator starts, outside latency-critical loops and before any stream capture. Later calls
 * allocate nothing. All calls share the array: calls that overlap on the GPU race and must be
 * serialised by the caller. */
fmm_status fmm_direct_B_noalloc(const float* xyz, const float* w, const float* J, int64_t n, const float* tgt,
                                int64_t m, double current, float* out_B, void* stream);

/* The reference's translation seam, kernels::translateAll* (FMM/FMMGPU/translation_algorithms.hpp:13-61),
 * plan-free, on the current device. Element type: float (precision FMM_FP32) or double (FMM_FP64),
 * matching the reference's `real`. on_device != 0: every pointer is device memory and the call only
 * queues work on `stream`; otherwise host memory, staged through stream-ordered allocations, and the
 * call waits for the result.
 *
 * fmm_translate_all <- translateAllCPU / translateAllGPU (translation_algorithms.hpp:13-25): for each
 * of `count` items, result[i] = M2M of the vector expansion expansions[i] ((order+1)^2 x 3 reals,
 * Vector3 AoS) by the real regular harmonics harmonics[i] ((order+1)^2 reals), with the reference's
 * real-form arithmetic (MultipoleTranslator::translateMultipole, multipole_translator.cpp:34-109).
 * All degrees 0..order are written (the reference's translateAllGPU leaves degree `order` unwritten,
 * translation_algorithms_gpu.cu:45-48; its translateAllCPU writes it). order <= 32. */
fmm_status fmm_translate_all(void* result, const void* harmonics, const void* expansions, int64_t count, int order,
                             int precision, int on_device, void* stream);
/* <- translateAllCPUMatrixBLAS / translateAllGPUMatrixCuBLAS (translation_algorithms.hpp:41-61): with
 * L = (order+1)^2, result (count x L) = a (count x L) * b (L x L), row-major, which is the reference's
 * column-major C = B * A. `batch` products share b: a and result hold `batch` consecutive count x L
 * blocks (the RealMatrix overload, three components, is batch = 3). batch <= 65535. */
fmm_status fmm_translate_all_matrix(void* result, const void* a, const void* b, int64_t count, int order,
                                    int64_t batch, int precision, int on_device, void* stream);
/* <- translateAllCPUMatrix / translateAllGPUMatrix (translation_algorithms.hpp:27-39): the same product
 * in complex arithmetic, elements (re, im) pairs (cuComplex / cuDoubleComplex layout). The reference's
 * GPU version launches a kernel whose body is commented out (kernels.cu:87-121) and returns zeros; this
 * computes what its CPU twin computes (math::multMatricesAsVectors, math.hpp:84-105). */
fmm_status fmm_translate_all_matrix_complex(void* result, const void* a, const void* b, int64_t count, int order,
                                            int precision, int on_device, void* stream);

/* Quadrature sources from the reference's tetrahedral torus, generated on the current device (the reference
 * builds them on the host: Torus::buildHexahedra and the split of each hexahedron into five tetrahedra,
 * FMM/FMMGPU/torus.cpp:52-117, then math::tetrahedraToQuadratures, integration.cpp:34-42,163-187): a torus of
 * square cross-section (side section_width, centre line of radius `radius`, axis z) cut into
 * n_length x n_width x n_height hexahedra, five tetrahedra each, and the basis rule rule_x[3k] (points on the
 * unit tetrahedron), rule_w[k] (k <= 64; the reference reads its Keast rule from files,
 * basis_quadratures.cpp:12-101) mapped into every tetrahedron: x = a + (b - a) u + (c - a) v + (d - a) w,
 * weight = volume x w_i. Outputs xyz[3 T k] and w[T k], T = 5 n_length n_width n_height, tetrahedron-major, in
 * `precision` (FMM_FP32 or FMM_FP64); device pointers with on_device != 0 (the call only queues work on
 * `stream`: pass them to fmm_set_sources with on_device = 1), host memory otherwise. */
fmm_status fmm_torus_quadratures(double radius, double section_width, int n_length, int n_width, int n_height,
                                 const double* rule_x, const double* rule_w, int k, int precision, void* xyz, void* w,
                                 int on_device, void* stream);

/* kernels::addVectors (FMMCUDADLL/kernel_callers.hpp:7-9): c = a + b for host arrays of n floats. */
fmm_status fmm_add_vectors(const float* a, const float* b, float* c, int64_t n);

const char* fmm_last_error_string(void);
const char* fmm_version(void);

#ifdef __cplusplus
}
#endif

#endif /* FMMCUDA_H */
