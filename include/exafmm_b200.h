/* exafmm_b200.h -- C ABI of the B200-native Laplace FMM (libexafmm_b200.so).
 *
 * Drop-in boundary for the exafmm-dev single-node FMM hot path.  Every entry point takes
 * plain pointers and sizes, returns an int status (FMM_OK = 0), and is re-entrant per
 * solver handle.  The reference has no return codes (assert/exit, include/macros.h:10-14);
 * here failures come back as status codes with a message from fmm_b200_last_error().
 *
 * Reference interfaces each group replaces:
 *   fmm_b200_build_tree     BoundBox::getBounds (include/bound_box.h:76-88) +
 *                           BuildTree::buildTree (include/build_tree_tbb.h:365-374, or
 *                           include/build_tree_omp.h:216-262 with FMM_TREE_UNIFORM)
 *   fmm_b200_upward_pass    UpDownPass::upwardPass (include/up_down_pass.h:119-132)
 *   fmm_b200_traverse       Traversal::dualTreeTraversal (include/traversal.h:240-264),
 *                           applying kernel::M2L / kernel::P2P (include/kernel.h:6-14)
 *   fmm_b200_downward_pass  UpDownPass::downwardPass (include/up_down_pass.h:135-148)
 *   fmm_b200_solve_*        the examples/serial.cxx:46-60 sequence in one call
 *   FMM_Init/FMM_Partition/FMM_Coulomb/FMM_Finalize   wrappers/gromacs.cxx:28-162
 *   fmm_init_/fmm_partition_/fmm_coulomb_/fmm_finalize_ wrappers/charmm.cxx:31-202
 *
 * Body and result arrays in the working precision are 4-vectors: bodies (x, y, z, q),
 * results (phi, dphi/dx, dphi/dy, dphi/dz) per unit target charge, in the caller's body
 * order (the reference's TRG after downwardPass, scattered back by IBODY).
 */
#ifndef EXAFMM_B200_H
#define EXAFMM_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define FMM_OK 0
#define FMM_ERR_INVALID 1        /* bad argument or configuration */
#define FMM_ERR_CUDA 2           /* CUDA runtime error (message in fmm_b200_last_error) */
#define FMM_ERR_NOT_SUPPORTED 3  /* e.g. periodic images with separate target/source sets */
#define FMM_ERR_NO_MEMORY 4      /* device allocation failed */
#define FMM_ERR_STATE 5          /* stage called out of order */
#define FMM_ERR_NO_DEVICE 6      /* no CUDA device / kernels not built for it */
#define FMM_ERR_DEVICE 7         /* a device-side check failed (capacity, depth) */

/* expansion basis: the reference's -DSpherical / -DCartesian (Makefile.include:37-41) */
#define FMM_SPHERICAL 0
#define FMM_CARTESIAN 1
/* working precision: FP32 expansions with compensated potential/gradient accumulation
 * (the reference's float real_t + -DKAHAN), or FP64 throughout (-DFP64) */
#define FMM_FP32 0
#define FMM_FP64 1

typedef struct fmm_b200_config {
  int basis;       /* FMM_SPHERICAL or FMM_CARTESIAN */
  int P;           /* expansion order: EXPANSION (include/types.h:38) */
  double theta;    /* opening angle (include/args.h:98, -t) */
  int ncrit;       /* bodies per leaf (include/args.h:98, -c) */
  int nspawn;      /* 2x2 split threshold of the traversal (include/args.h:98, -s) */
  int use_rmax;    /* include/args.h:99 (-x) */
  int use_ropt;    /* include/args.h:99 (-o) */
  int precision;   /* FMM_FP32 or FMM_FP64 */
  double eps2;     /* softening squared (Traversal::eps2; see fmm_b200_config note) */
  int images;      /* periodic image levels (Traversal::images, include/traversal.h:21):
                    * 0 open boundary; k > 0: the 27 nearest copies of the box through the
                    * tree and k - 1 levels of 3x3x3 super-cells of copies through the root
                    * multipole (traversePeriodic); either basis */
  int device;      /* CUDA device ordinal */
  double cycle;    /* period of the box when images > 0 (dualTreeTraversal's cycle) */
  int mutual;      /* dualTreeTraversal's mutual flag (include/traversal.h:240): each unordered
                    * cell pair visited once and applied both ways (open boundary, one tree);
                    * the device evaluates both ways from the target side, so the results are
                    * the reference's mutual ones to rounding */
  int tree;        /* FMM_TREE_ADAPTIVE: BuildTree of include/build_tree_tbb.h (the -DTBB
                    * build); FMM_TREE_UNIFORM: BuildTree of include/build_tree_omp.h (an
                    * OpenMP build without TBB, include/build_tree.h:12-13), every leaf at depth
                    * 1 + int(log(N / ncrit) / ln 2 / 3); one tree per call (batches and
                    * separate target/source sets return FMM_ERR_NOT_SUPPORTED), depth <= 10 */
} fmm_b200_config;

/* tree builders (fmm_b200_config.tree) */
#define FMM_TREE_ADAPTIVE 0
#define FMM_TREE_UNIFORM 1

typedef struct fmm_b200_solver fmm_b200_solver;

/* phase timings (milliseconds of device time, CUDA events on the solver's stream), in the
 * reference's logger phase order (include/logger.h:87-106 call sites) */
#define FMM_PHASE_BOUNDS 0
#define FMM_PHASE_TREE 1
#define FMM_PHASE_UPWARD 2
#define FMM_PHASE_TRAVERSE 3   /* list construction */
#define FMM_PHASE_M2L 4
#define FMM_PHASE_P2P 5
#define FMM_PHASE_DOWNWARD 6
#define FMM_PHASE_TOTAL 7
#define FMM_NUM_PHASES 8

/* ---- lifecycle --------------------------------------------------------------------- */
/* Defaults: spherical, P = 10, theta = 0.4, ncrit = 64, nspawn = 1000, use_rmax = 1,
 * use_ropt = 1, FP32, eps2 = 0, images = 0, device 0, adaptive tree. */
int fmm_b200_default_config(fmm_b200_config* cfg);
int fmm_b200_create(const fmm_b200_config* cfg, fmm_b200_solver** out);
int fmm_b200_destroy(fmm_b200_solver* s);
/* Work is issued on this stream (a cudaStream_t; NULL = the legacy default stream). */
int fmm_b200_set_stream(fmm_b200_solver* s, void* stream);
/* A handle grows its device arrays when a solve needs more, and keeps the buffers it grew
 * out of instead of freeing them during the solve (cudaFree synchronises the whole device,
 * which would stall the caller's other streams); they add up to at most the arrays'
 * final size and are freed with the handle.  fmm_b200_trim frees them now: a device-wide
 * synchronisation, for a moment when the device is idle.  No reference counterpart. */
int fmm_b200_trim(fmm_b200_solver* s);
/* Periodic boundary of the next traversals: image levels and period (the arguments the
 * reference passes to Traversal() and dualTreeTraversal(); include/traversal.h:216-264). */
int fmm_b200_set_periodic(fmm_b200_solver* s, int images, double cycle);
/* mutual flag of the next traversals (dualTreeTraversal's mutual argument) */
int fmm_b200_set_mutual(fmm_b200_solver* s, int mutual);
/* One solve over nparts GPUs, one handle per GPU, every handle given the same bodies: the
 * handle computes the results of part `part` only.  After the tree build its bodies (tree
 * order) are cut into nparts ranges of about n / nparts bodies, each cut moved down to the
 * start of the leaf that holds it; the traversal keeps the pairs whose target cell holds
 * bodies of this part (exactly the whole traversal's pairs for those targets), M2L and P2P
 * run on them, L2L on the cells that hold bodies of this part, L2P on this part's bodies,
 * and the other bodies' results are 0.  The tree and the upward pass are computed on every
 * handle.  The sum of the nparts results (an all-reduce, or a reduce-scatter to the bodies'
 * owners) is the one-GPU solve's result, bit for bit.  Whole single solves with an open or
 * periodic boundary (FMM_ERR_NOT_SUPPORTED for batches, separate target/source sets and the
 * mutual traversal).  nparts = 1 (the default) computes every body.  The reference spreads
 * a solve over MPI ranks by an ORB partition of the bodies plus the exchange of a local
 * essential tree (include/partition.h:69-195, include/tree_mpi.h:225-369); this replaces the
 * exchange by replicated bodies and tree, for the GPUs of one node, each with room for all
 * the bodies.  The single-operator calls (fmm_b200_kernel_*) ignore the partition. */
int fmm_b200_set_partition(fmm_b200_solver* s, int part, int nparts);
/* The handle's part and nparts, and after a solve this part's bodies [begin, end) in tree
 * order (0, n when nparts = 1); any pointer may be NULL. */
int fmm_b200_get_partition(fmm_b200_solver* s, int* part, int* nparts, int* body_begin,
                           int* body_end);
/* Message of the last failure on this handle (or of the last failed create if s is NULL). */
const char* fmm_b200_last_error(const fmm_b200_solver* s);
/* Which P values were compiled for a basis: writes up to cap values, returns the count. */
int fmm_b200_supported_orders(int basis, int* orders, int cap);

/* ---- whole solve --------------------------------------------------------------------- */
/* Bodies and results in device memory (4-vectors in the working precision, caller order).
 * Stream-ordered; returns once the work is queued (plus the few host reads the level
 * structure needs). */
int fmm_b200_solve_device(fmm_b200_solver* s, int n, const void* d_bodies, void* d_trg);
/* Host double arrays as in FMM_Coulomb (wrappers/gromacs.cxx:104-162): x interleaved
 * (3n), q (n); p (n) and f (3n) receive phi and grad phi.  Copies in and out inside the
 * call; synchronous. */
int fmm_b200_solve_host(fmm_b200_solver* s, int n, const double* x, const double* q,
                        double* p, double* f);

/* ---- batches of independent solves --------------------------------------------------- *
 * nsolves solves with counts[s] bodies each, bodies concatenated in solve order (device
 * 4-vectors or host doubles as above), results in the same layout.  The solves share one
 * tree build, traversal and set of kernel launches ("forest": one root per non-empty
 * solve, cells of a solve contiguous, no interaction across solves); every solve's result
 * is bitwise the one it gets alone.  All solves use the handle's configuration.
 * No reference counterpart: the reference solves one system per call. */
int fmm_b200_solve_batch_device(fmm_b200_solver* s, int nsolves, const int* counts,
                                const void* d_bodies, void* d_trg);
int fmm_b200_solve_batch_host(fmm_b200_solver* s, int nsolves, const int* counts,
                              const double* x, const double* q, double* p, double* f);
int fmm_b200_set_bodies_batch_device(fmm_b200_solver* s, int nsolves, const int* counts,
                                     const void* d_bodies);
/* Roots after the tree build: their count, first cell, and solve index. */
int fmm_b200_get_roots(fmm_b200_solver* s, int* nroots, int* root_cells, int* root_solves);

/* ---- stages (the reference's class methods) ------------------------------------------ */
int fmm_b200_set_bodies_host(fmm_b200_solver* s, int n, const double* x, const double* q);
int fmm_b200_set_bodies_device(fmm_b200_solver* s, int n, const void* d_bodies);
int fmm_b200_build_tree(fmm_b200_solver* s);
int fmm_b200_upward_pass(fmm_b200_solver* s);
int fmm_b200_traverse(fmm_b200_solver* s);
int fmm_b200_downward_pass(fmm_b200_solver* s);
int fmm_b200_get_trg_host(fmm_b200_solver* s, double* trg);   /* 4n, caller order */
int fmm_b200_get_trg_device(fmm_b200_solver* s, void* d_trg); /* 4n working precision */

/* ---- introspection (tree, lists, expansions; host copies) ----------------------------- */
int fmm_b200_num_cells(fmm_b200_solver* s, int* num_cells, int* max_level);
/* Cells in the reference layout (include/types.h:79-92, include/build_tree_tbb.h:250-294):
 * X is 3 per cell; R is the current radius (after build: R0 / 2^level; after the upward
 * pass: the MAC radius). */
int fmm_b200_get_cells(fmm_b200_solver* s, int* iparent, int* ichild, int* nchild,
                       int* ibody, int* nbody, unsigned long long* icell, int* level,
                       double* X, double* R);
/* Original index (IBODY) of each body in tree order. */
int fmm_b200_get_order(fmm_b200_solver* s, int* ibody);
/* Root box: X0[3], R0 (BuildTree::bounds2box, include/build_tree_tbb.h:298-310). */
int fmm_b200_get_box(fmm_b200_solver* s, double* x0r0);
/* which = 0: multipoles M, 1: locals L.  Spherical: NTERM (re, im) pairs per cell;
 * Cartesian: NTERM reals per cell. */
int fmm_b200_get_expansion(fmm_b200_solver* s, int which, double* out);
/* Interaction lists of the last traversal: cell pairs packed (target << 32) | source |
 * image << 27, sorted; image is 0 without periodic images, else the source tree's shift
 * (ix, iy, iz) cycle, |i| <= 1, coded 9 d(ix) + 3 d(iy) + d(iz) with d(0) = 0, d(1) = 1,
 * d(-1) = 2.  Body-pair counts are the sum of target x source body counts. */
int fmm_b200_num_lists(fmm_b200_solver* s, long long* num_m2l, long long* num_p2p,
                       long long* p2p_body_pairs);
int fmm_b200_get_lists(fmm_b200_solver* s, long long* m2l, long long* p2p);
int fmm_b200_get_timings(fmm_b200_solver* s, double* ms); /* FMM_NUM_PHASES values */

/* ---- single operators: namespace kernel (include/kernel.h:6-14) --------------------------
 * The reference's kernel plugin interface, kernel::P2M / M2M / M2L / L2L / L2P / P2P, which
 * examples/kernel.cxx:23-92, the up/down passes and the traversal call one cell (pair) at a
 * time, as calls over lists of cells of a handle: the cells of its last tree build, or cells
 * set up by hand with fmm_b200_kernel_set_cells over the bodies of fmm_b200_set_bodies_* in
 * their given order.  Each call runs the handle's own kernels (its basis, order P and
 * precision) and accumulates as the reference does: P2M / M2M add to the cells' M, M2L /
 * L2L to their L, L2P / P2P to the bodies' targets (phi, grad phi per unit target charge;
 * the reference's TRG carries the target charge until L2P divides by it).  Multipoles are
 * unnormalised (the reference's non-MASS build).  Entries of one call run concurrently, so
 * a call must not list a cell with its child (M2M) or parent (L2L), the same cell twice
 * (P2M, M2M, L2L, L2P), or target cells whose bodies overlap (L2P, P2P); such lists and any
 * index out of range return FMM_ERR_INVALID before the device is touched.  Pairs carry an
 * optional image code per pair (NULL: no shift; the code of fmm_b200_get_lists, shift
 * (ix, iy, iz) times the handle's period) and the mutual flag (each pair of two different
 * cells also applied in reverse).  The calls leave the expansions readable
 * (fmm_b200_get_expansion) and the handle's interaction lists stale. */
/* Cells by hand: X (3 per cell) and R, the body range [ibody, ibody + nbody) of each cell,
 * children [ichild, ichild + nchild) and parent iparent (include/types.h:79-94); M, L and
 * the targets start at zero. */
int fmm_b200_kernel_set_cells(fmm_b200_solver* s, int ncells, const double* X, const double* R,
                              const int* ibody, const int* nbody, const int* ichild,
                              const int* nchild, const int* iparent);
/* which = 0: M, 1: L, in the fmm_b200_get_expansion layout; NULL sets zero */
int fmm_b200_kernel_set_expansion(fmm_b200_solver* s, int which, const double* in);
/* targets of the bodies in cell order (4 per body); NULL sets zero */
int fmm_b200_kernel_set_trg(fmm_b200_solver* s, const double* trg);
int fmm_b200_kernel_get_trg(fmm_b200_solver* s, double* trg);
/* kernel::P2M(C) for each listed cell: M += sum of q Y(body - X) (LaplaceSphericalCPU.cxx:103-118) */
int fmm_b200_kernel_p2m(fmm_b200_solver* s, int n, const int* cells);
/* kernel::M2M(Ci, C0): M += the cell's children's multipoles shifted to its centre (:120-147) */
int fmm_b200_kernel_m2m(fmm_b200_solver* s, int n, const int* cells);
/* kernel::M2L(Ci, Cj, Xperiodic, mutual): L of ci[k] += M of cj[k] translated (:149-191) */
int fmm_b200_kernel_m2l(fmm_b200_solver* s, int n, const int* ci, const int* cj,
                        const int* image, int mutual);
/* kernel::L2L(Ci, C0): L += the parent's local expansion shifted to the cell's centre (:193-224) */
int fmm_b200_kernel_l2l(fmm_b200_solver* s, int n, const int* cells);
/* kernel::L2P(Ci): the cell's bodies' targets += its local expansion evaluated (:226-256) */
int fmm_b200_kernel_l2p(fmm_b200_solver* s, int n, const int* cells);
/* kernel::P2P(Ci, Cj, eps2, Xperiodic, mutual) and the self form P2P(C, eps2) (ci[k] ==
 * cj[k]): targets of ci[k]'s bodies += the field of cj[k]'s bodies, r^2 == 0 pairs skipped
 * (kernels/LaplaceP2PCPU.cxx:4-331) */
int fmm_b200_kernel_p2p(fmm_b200_solver* s, int n, const int* ci, const int* cj,
                        const int* image, int mutual, double eps2);

/* ---- separate target and source sets ----------------------------------------------------
 * Targets (nt, with charges qt that shape their own tree's radii) and sources (ns) in two
 * trees, both upward passes, dualTreeTraversal(cells, jcells) from the target root against
 * the source root, the targets' downward pass.  common_box = 1: both trees on the box of
 * the two sets' common bounds (examples/serial.cxx with IneJ, :30-55); 0: each tree on its
 * own bodies' box (wrappers/petiga.cxx:134-139).  p, f (host) or d_trg (device 4-vectors)
 * receive the targets' potential and gradient per unit target charge, in input order.
 * Open boundary only (images > 0: FMM_ERR_NOT_SUPPORTED).  Lists and cells of the last call
 * are the two trees' (source cells after the target tree's, from the second root of
 * fmm_b200_get_roots). */
int fmm_b200_solve_ij_host(fmm_b200_solver* s, int nt, const double* xt, const double* qt,
                           int ns, const double* xs, const double* qs, int common_box, double* p,
                           double* f);
int fmm_b200_solve_ij_device(fmm_b200_solver* s, int nt, const void* d_targets, int ns,
                             const void* d_sources, int common_box, void* d_trg);

/* ---- autotuning ------------------------------------------------------------------------
 * Picks ncrit (bodies per leaf, which sets the split between P2P and M2L work) for the
 * bodies last given to the handle (fmm_b200_set_bodies_* or a solve): every candidate
 * solves them `repeats` times after one untimed solve; the median device time of each goes
 * to times_ms[i] (may be NULL) and the fastest becomes the handle's ncrit (*best_ncrit).
 * Results depend on ncrit only through the tree (same method error).  No reference
 * counterpart (the reference takes ncrit from the command line, include/args.h:98). */
int fmm_b200_autotune_ncrit(fmm_b200_solver* s, const int* candidates, int ncand, int repeats,
                            int* best_ncrit, double* times_ms);
/* Picks the P2P kernel's threads per target group (lanes that share one target body) on the
 * interaction lists of the handle's last solve: candidate i gives a target 4 lanes in leaves
 * of at most lanes4_max[i] bodies, 2 lanes in leaves of at most lanes2_max[i], else 1
 * (0 <= lanes4_max <= 8, lanes4_max <= lanes2_max <= 16; the default is 8 / 16).  Each runs the
 * P2P `repeats` times after one untimed run; the median device time goes to times_ms[i]
 * (may be NULL) and the fastest becomes the handle's (index in *best).  The split of a
 * target's sources over its lanes changes only the rounding of its sums.  The handle must
 * solve again before its results are read.  No reference counterpart. */
int fmm_b200_autotune_p2p(fmm_b200_solver* s, const int* lanes4_max, const int* lanes2_max,
                          int ncand, int repeats, int* best, double* times_ms);

/* ---- serving: continuous batching of independent solves ------------------------------ *
 * A server owns nworkers worker threads (one CUDA stream and one solver handle per order
 * each) and a scheduler that batches pending requests of equal order P, in arrival order,
 * within hbm_budget_bytes of estimated device memory, max_batch solves and 2^21 bodies
 * per batch (a larger request rides alone).  Each worker holds pinned host staging for
 * 2^21 bodies (128 MB) from the start, and sizes each new handle (the first request of an
 * order on a worker) with two synthetic batches of 2^21 bodies before it takes requests, so
 * that later passes rarely allocate.  Batches on different workers overlap on the device;
 * a request arriving while batches run joins the next batch a worker takes.  cfg supplies
 * basis, theta, ncrit, nspawn, precision and device (its P need not be compiled for the
 * basis); P comes with each request.  submit copies the inputs; wait blocks
 * until the request is done, copies p (n) and f (3n), and reports its latency (submit to
 * done) and queueing time (submit to batch start) in seconds.  A request whose estimate
 * exceeds the whole budget is rejected with FMM_ERR_NO_MEMORY.  destroy drains the queue.
 * No reference counterpart. */
typedef struct fmm_b200_server fmm_b200_server;
int fmm_b200_server_create(const fmm_b200_config* cfg, double hbm_budget_bytes, int nworkers,
                           int max_batch, fmm_b200_server** out);
int fmm_b200_server_submit(fmm_b200_server* srv, int n, const double* x, const double* q,
                           int P, long long* request_id);
/* Opening angle for the requests of order P submitted from now on (0 < theta < 1; else the
 * configuration's theta): a lower order needs a smaller angle for the same accuracy, e.g.
 * rel-L2 <= 1e-4 of potential and gradient on zero-net-charge cubes of 1e3..1e6 bodies
 * needs theta <= 0.22 at P = 6, 0.30 at P = 8, 0.35 at P = 10 with a margin of two.  Only
 * requests of equal order and angle share a batch. */
int fmm_b200_server_set_theta(fmm_b200_server* srv, int P, double theta);
int fmm_b200_server_poll(fmm_b200_server* srv, long long request_id, int* done);
int fmm_b200_server_wait(fmm_b200_server* srv, long long request_id, double* p, double* f,
                         double* latency_s, double* queue_s);
int fmm_b200_server_stats(fmm_b200_server* srv, long long* completed, long long* bodies,
                          long long* batches, int* pending);
/* Worker seconds summed over all batches so far: copying requests into the pinned staging
 * buffer, inside the batched solve (host<->device copies included), copying results out. */
int fmm_b200_server_profile(fmm_b200_server* srv, double* stage_s, double* solve_s,
                            double* unstage_s);
/* Free the device buffers the workers' handles have grown out of (fmm_b200_trim on each):
 * waits until no batch runs and holds new batches back meanwhile (a device-wide
 * synchronisation: for a quiet moment).  The server never does this by itself, so that a
 * burst that arrives while it would run is not held up; the buffers kept add up to at most
 * the handles' arrays, and destroy frees everything. */
int fmm_b200_server_trim(fmm_b200_server* srv);
int fmm_b200_server_destroy(fmm_b200_server* srv);

/* ---- utilities ----------------------------------------------------------------------- */
/* FP64 direct sum on the GPU: Traversal::direct + normalize (include/traversal.h:304-337)
 * with double accumulation.  Targets xt (3 nt), sources xs (3 ns) with charges qs; out
 * receives 4 nt values (phi, grad phi) per unit target charge; pairs with r^2 + eps2 == 0
 * are skipped.  Synchronous; a failure's message is in fmm_b200_last_error(NULL). */
int fmm_b200_direct(int device, int nt, const double* xt, int ns, const double* xs,
                    const double* qs, double eps2, double* out);
/* fmm_b200_direct without any device allocation: same arguments, kernel and (bitwise)
 * result, with the device staging buffers in a static device array of 3.75 MiB (7 nt + 4 ns
 * doubles), which every GPU that loads this library holds until the process exits, instead
 * of a cudaMalloc/cudaFree per call.  For callers that cannot allocate device memory while
 * they run: those whose device memory is all held by their own pool allocator, and those
 * that must not take the device-wide synchronisation that cudaMalloc/cudaFree imply while
 * other streams of theirs are busy.  No counterpart in the reference.
 * Limits: nt <= FMM_DIRECT_NOALLOC_MAX_TARGETS and ns <= FMM_DIRECT_NOALLOC_MAX_SOURCES;
 * larger sizes return FMM_ERR_INVALID, with the limits in fmm_b200_last_error(NULL), before
 * the device is touched.  Every call clears that message first, so it describes this call's
 * failure or is empty after a success.  The first call on each device does the set-up: it looks up the
 * array's address (cudaGetSymbolAddress, with that device current), which may load the
 * library's device code; make that first call before any stream capture begins on the
 * device.  Nothing in the array has to start at zero: a call copies in every input it reads
 * and writes every output it returns.  All calls on one device share the array and it keeps
 * the last call's contents: calls that overlap on the same GPU (from several host threads)
 * race on it, and the caller must serialise them.  Synchronous: the result is in `out` when
 * the call returns. */
#define FMM_DIRECT_NOALLOC_MAX_TARGETS 32768
#define FMM_DIRECT_NOALLOC_MAX_SOURCES 65536
int fmm_b200_direct_noalloc(int device, int nt, const double* xt, int ns, const double* xs,
                            const double* qs, double eps2, double* out);
/* FP32 FMA throughput of the device in TFLOP/s (independent FMA chains on every SM): the
 * roofline denominator of the FP32-pipe kernels (M2L, P2P).  No reference counterpart. */
int fmm_b200_fp32_peak(int device, double* tflops);
/* Number of this library's own kernel launches so far (library calls such as CUB sorts are
 * not counted).  No reference counterpart. */
long long fmm_b200_kernel_launches(void);
/* Number of device allocations (cudaMalloc) the solver handles have made so far: a handle
 * grows its arrays the first time a solve needs more, and each growth synchronises the
 * device.  No reference counterpart. */
long long fmm_b200_device_allocations(void);

/* ---- reference wrapper ABI (single GPU, single rank) ----------------------------------
 * (Left out when EXAFMM_B200_NO_GROMACS_ABI is defined: the PetIGA wrapper library,
 * include/exafmm_b200_petiga.h, reuses the names FMM_Init / FMM_Partition / FMM_Finalize.)
 * FMM_Init: the gromacs wrapper's fixed parameters (ncrit 32, nspawn 1000, theta 0.4,
 * use_rmax, use_ropt, eps2 0, wrappers/gromacs.cxx:28-56) on the spherical basis at
 * EXAFMM_B200_P (default 10) in FP32, with `images` periodic image levels of the box of
 * side `cycle` that each FMM_Coulomb call passes. */
#ifndef EXAFMM_B200_NO_GROMACS_ABI
void FMM_Init(int images);
void FMM_Finalize(void);
#ifdef __cplusplus
void FMM_Partition(int& n, int* index, double* x, double* q, double cycle);
#else
void FMM_Partition(int* n, int* index, double* x, double* q, double cycle);
#endif
void FMM_Coulomb(int n, double* x, double* q, double* p, double* f, double cycle);
#endif

/* Fortran ABI of the CHARMM wrapper (wrappers/charmm.cxx:31-202), single rank: bodies
 * with icpumap[i] == 1 are solved and p, f accumulate TRG * q * 332.0716. */
void fmm_init_(int* images, double* theta, int* verbose);
void fmm_finalize_(void);
void fmm_partition_(int* nglobal, int* icpumap, double* x, double* q, double* xold,
                    double* cycle);
void fmm_coulomb_(int* nglobal, int* icpumap, double* x, double* q, double* p, double* f,
                  double* cycle);

#ifdef __cplusplus
}
#endif
#endif
