/*
 * coulombo_lattice.h -- C ABI of the B200 Coulomb-integral library (libcoulombo_lattice.so).
 *
 * The reference (Coulombo-Lattice, Rozanski & Zielinski, Comput. Phys. Commun. 287 (2023)
 * 108693) has no plugin or FFI layer: its compute seam is the C++ class CoulombCalculator
 * fed by Product::map and Interaction::map inside one executable.  Each entry point below
 * names the reference interface it replaces (path:line within the reference project).
 *
 * Conventions
 *   - Every call returns 0 on success and a non-zero CL_ERR_* code on failure; the message
 *     is then available from cl_last_error() (thread-local).  No C++ exception crosses this
 *     boundary and no call aborts the process.
 *   - All array arguments are caller-owned HOST buffers; the library copies them to the GPU.
 *   - Grids are x-fastest: cell index = (iz*ny + iy)*nx + ix (run-tests.cpp:169-175).
 *   - Complex values are interleaved {re, im} doubles.
 *   - One context per host thread; a context is bound to the CUDA device that was current
 *     when it was created.
 */
#ifndef COULOMBO_LATTICE_H
#define COULOMBO_LATTICE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define CL_OK              0
#define CL_ERR_ARGUMENT    1  /* invalid argument (reference: std::logic_error / runtime_error) */
#define CL_ERR_STATE       2  /* call out of order, e.g. calculate() before prepare() */
#define CL_ERR_CUDA        3  /* CUDA runtime failure or no usable GPU */
#define CL_ERR_MEMORY      4  /* device or host allocation failed */
#define CL_ERR_UNSUPPORTED 5  /* size outside what the kernels handle (e.g. not 2*3*5-smooth) */
#define CL_ERR_TIMEOUT     6  /* a bounded device-side wait gave up */

/* precision / algorithm forms */
#define CL_MODE_FP64_PLAIN   0  /* all-FP64: 8 rounds of FFT -> x Ghat -> iFFT, real-space dot */
#define CL_MODE_FP32_ROUNDS  1  /* the same 8 rounds with FP32 FFT stages; FP64 kernel, twiddles,
                                   round sum and reductions (split-precision tensor-core Gram) */
#define CL_MODE_FP32_FOURIER CL_MODE_FP32_ROUNDS /* former name of CL_MODE_FP32_ROUNDS */
/* The sub-lattice forms compute the same aperiodic convolution exactly, but per residue class of
 * the atoms' grid points modulo m (m = 4 or 2 per axis): each occupied class is a dense sub-grid
 * transformed with zero padding to 2n/m points per axis, and the classes are coupled once per
 * frequency by kernels built from the same Ghat.  For zinc-blende or diamond on the a/4 grid (8
 * of 64 classes) that is one eighth of the 8-round method's transform work.  The choice is made
 * when the states are loaded: a structure that occupies too many classes (or a grid size not
 * divisible by m) runs the 8-round method of the same precision.  The grid-level calls
 * (cl_prepare_grid ...) always run the 8 rounds.  cl_form_info reports what was chosen. */
#define CL_MODE_FP64_SUBLATTICE 2  /* all-FP64 sub-lattice form */
#define CL_MODE_FP32_SUBLATTICE 3  /* sub-lattice form with FP32 transforms; FP64 kernel and class
                                      kernels built in FP64 and rounded once; split-precision
                                      tensor-core reductions with FP64 accumulation */

typedef struct cl_ctx cl_ctx;

/* ---------------------------------------------------------------------------------------
 * Calculator life cycle
 * ------------------------------------------------------------------------------------- */

/* Create a calculator for an nx*ny*nz grid with step lengths (sx, sy, sz) in Angstrom.
 * Replaces CoulombCalculator::CoulombCalculator(const Dimension&) (src/CoulombCalculator.cpp:11-55)
 * together with the step argument of InteractionBase (src/Interaction.hpp:19-20).
 * Sizes must be products of 2, 3 and 5 (what Broadcaster::round4FFT produces,
 * src/Broadcaster.cpp:136-143). */
int cl_create(cl_ctx** out, int nx, int ny, int nz, double sx, double sy, double sz, int mode);

/* Release every device buffer of the context.  Safe on NULL. */
void cl_destroy(cl_ctx* ctx);

/* Message of the last failed call on this thread ("" if none). */
const char* cl_last_error(void);

/* ---------------------------------------------------------------------------------------
 * Coulomb kernel: Interaction::map + CoulombCalculator::initialize
 * ------------------------------------------------------------------------------------- */

/* G(r) = e^2/(4 pi eps0) / (eps(r) r) on the (nx+1)(ny+1)(nz+1) octant, G(0) = onsite (eV),
 * then Ghat = REDFT00 (3D DCT-I) / (8 nx ny nz).  tf_lattice <= 0 selects the simple model
 * (InteractionSimple, src/Interaction.cpp:8-14); tf_lattice > 0 the Thomas-Fermi-Resta model
 * (InteractionThomasFermi, src/Interaction.cpp:18-39), which requires dielectric > 1.
 * Replaces src/Interaction.hpp:32-51 and src/CoulombCalculator.cpp:57-103. */
int cl_set_kernel_coulomb(cl_ctx* ctx, double dielectric, double onsite, double tf_lattice);

/* Same as above for a caller-supplied octant G[(nx+1)(ny+1)(nz+1)] (x fastest): the
 * reference's custom-Interaction seam (run-tests.cpp:13-21 feeds one to CoulombCalculator). */
int cl_set_kernel_grid(cl_ctx* ctx, const double* G);

/* ---------------------------------------------------------------------------------------
 * Grid-level calculator (the reference's prepare/calculate state machine)
 * ------------------------------------------------------------------------------------- */

/* input = rho (nx*ny*nz complex), then prepare(): V = aperiodic G * rho by 8 rounds.
 * Replaces CoulombCalculator::input + prepare() (src/CoulombCalculator.hpp:48, .cpp:105-163). */
int cl_prepare_grid(cl_ctx* ctx, const double* rho);

/* input = rho2, then calculate(): out = sum_r V(r) rho2(r) (no conjugation), reusing the
 * last prepare.  Replaces CoulombCalculator::calculate() (src/CoulombCalculator.cpp:165-172). */
int cl_calculate_grid(cl_ctx* ctx, const double* rho2, double out[2]);

/* Copy the quasi-potential V of the last cl_prepare_grid (nx*ny*nz complex) to the host.
 * Replaces CoulombCalculator::potential() (src/CoulombCalculator.hpp:90-93). */
int cl_potential_grid(cl_ctx* ctx, double* V);

/* ---------------------------------------------------------------------------------------
 * Integral pipeline (FunctionCollection + Planner + the coulombo main loop)
 * ------------------------------------------------------------------------------------- */

/* Upload n_states LCAO states of n_atoms atoms x n_orb orbitals, coeff laid out
 * [state][atom][orbital]{re,im} (the file order of src/FunctionCollection.cpp:56-84), and
 * the grid cell of every atom (src/Broadcaster.cpp:76-87).  States are in input order,
 * holes first (coulombo.cpp:96-117).  Replaces FunctionCollection::appendFile and the
 * Broadcaster's coefficient scatter (src/FunctionCollection.cpp:86-89, src/Broadcaster.cpp:96-103). */
int cl_set_states(cl_ctx* ctx, int n_states, int n_holes, int64_t n_atoms, int n_orb,
                  const double* coeff, const int64_t* cells);

/* Compute n_int integrals spec[i] = (i1,i2,i3,i4), 1-based input indices, into
 * out[i] = {re, im} in eV.  Product indexing, conjugation flags, plan orientation and the
 * result conjugation follow the reference (src/Planner.hpp:71-144, src/Graph.hpp:49-91,
 * coulombo.cpp:186-209).  Replaces the whole "Computing requested integrals" phase. */
int cl_compute(cl_ctx* ctx, int64_t n_int, const int16_t* spec, double* out);

/* cl_set_states followed by cl_compute in one call, with the coefficient upload overlapped
 * with the transforms: the states are copied one at a time on a second stream, and each
 * group of left densities starts its pair densities and rounds as soon as its last state has
 * arrived.  Same arguments, results and errors as the two calls; the coefficient buffer is only
 * read during the call (pinned host memory lets the copies run asynchronously).  A cell list
 * identical to the previous call's is not sorted or uploaded again.  No reference counterpart:
 * the reference reads every file before computing (coulombo.cpp:99-117, 186-209). */
int cl_compute_states(cl_ctx* ctx, int n_states, int n_holes, int64_t n_atoms, int n_orb, const double* coeff,
                      const int64_t* cells, int64_t n_int, const int16_t* spec, double* out);

/* V of every state's own density |psi_s|^2 (real part) at every atom, out[state][atom].
 * Replaces the loop of potentials.cpp:137-158 (createSelfProducts, prepare,
 * extractAtomCellValues at src/FunctionCollection.cpp:122-131). */
int cl_potentials(cl_ctx* ctx, double* out);

/* Same as cl_compute restricted to the rounds kappa whose bit is set in round_mask
 * (bit 0 = kappa 0 ... bit 7 = kappa 7).  The integrals are sums over rounds
 * (CoulombCalculator.cpp:105-163 accumulates V_ += Ftemp per round), so partial results
 * of disjoint masks add up to cl_compute's: the unit of work a multi-GPU split hands each
 * rank before one all-reduce.  No reference counterpart (single-process decomposition of
 * the reference's prepare()). */
int cl_compute_rounds(cl_ctx* ctx, int64_t n_int, const int16_t* spec, int round_mask, double* out);

/* What the context runs for the loaded states: info[0] = 1 when the sub-lattice
 * decomposition is used (0: the 8 rounds), info[1] = m, info[2] = occupied classes S,
 * info[3] = 1 when the classes are the zinc-blende set (compiled mixing table), info[4..6] =
 * transform lengths per axis (2n/m), info[7] = class kernels stored per frequency.  No reference
 * counterpart (the reference always runs the 8 rounds, CoulombCalculator.cpp:105-163). */
int cl_form_info(cl_ctx* ctx, int info[8]);

/* Same as cl_compute for one shard of the request: the prepared (left) densities of the plan, in
 * ascending product order, are dealt round-robin to n_shards shards, and out[i] holds integral i
 * when its left density belongs to shard `shard`, zero otherwise.  The shards' outputs add up to
 * cl_compute's, so n_shards GPUs (one process each) run one shard each and combine them with one
 * all-reduce (sum) of out: the multi-GPU unit of both forms (the sub-lattice forms have no
 * rounds).  Right densities are formed on every shard.  No reference counterpart: the reference
 * splits each grid over MPI ranks and reduces every calculate() (CoulombCalculator.cpp:165-172). */
int cl_compute_shard(cl_ctx* ctx, int64_t n_int, const int16_t* spec, int shard, int n_shards, double* out);

/* Device time in milliseconds of the phases of the last cl_compute / cl_potentials:
 * t[0] pair densities, t[1] transforms (all rounds), t[2] reductions, t[3] total. */
int cl_last_timings(cl_ctx* ctx, double t[4]);

/* Choices of the autotuner (process-wide): one text line per tuned pass, grid shape and
 * precision -- the radix split, lines per block and tile layout kept, with the per-launch time of the
 * tuning sample next to the default variant's.  Writes at most len bytes (NUL-terminated) to
 * buf when buf is non-null; *needed (if non-null) receives the full size.  No reference
 * counterpart: the reference plans its FFTs with FFTW_MEASURE / FFTW_ESTIMATE
 * (CoulombCalculator.cpp:17-39).  CL_AUTOTUNE=0 in the environment disables tuning;
 * CL_TUNE_FILE=<path> loads earlier choices from that file and appends new ones to it. */
int cl_autotune_report(char* buf, int64_t len, int64_t* needed);

/* Per-kernel timing with CUDA events recorded on the context's stream around every launch.
 * Classes: */
#define CL_KCLASS_DENSITY   0  /* pair densities at atoms */
#define CL_KCLASS_XFWD      1  /* scatter + phase + FFT along x */
#define CL_KCLASS_YPASS     2  /* FFT along y (both directions) */
#define CL_KCLASS_ZPASS     3  /* FFT along z, x Khat, inverse FFT along z */
#define CL_KCLASS_XINV      4  /* inverse FFT along x + phase + accumulate V at atoms */
#define CL_KCLASS_GRAM      5  /* real-space reductions: FP64 Gram (plain) or tensor-core Gram (FP32 form) */
#define CL_KCLASS_KERNEL    6  /* Coulomb kernel octant, DCT-I, folded kernels */
#define CL_KCLASS_GRAM_SPLIT 7 /* TF32 hi/lo operand split of the tensor-core Gram (FP32 form) */
#define CL_KCLASS_ROUND_SUM 8  /* x phase_kappa and the FP64 sum of the rounds at the atoms */
#define CL_NUM_KCLASS       10
/* enable != 0 starts recording (and clears the counters); 0 stops. */
int cl_set_profiling(cl_ctx* ctx, int enable);
/* Accumulated device milliseconds, launches and algorithmic bytes (the minimum HBM
 * traffic of each launch's work, see the kernel notes) per class since profiling started. */
int cl_kernel_profile(cl_ctx* ctx, double ms[CL_NUM_KCLASS], int64_t launches[CL_NUM_KCLASS],
                      double bytes[CL_NUM_KCLASS]);

/* ---------------------------------------------------------------------------------------
 * Prepared requests and graph-captured batches of independent structures
 * ------------------------------------------------------------------------------------- */

typedef struct cl_request cl_request;
typedef struct cl_batch cl_batch;

/* A request prepared once: the plan of n_int integrals (as for cl_compute), its device
 * buffers and its pinned result buffer.  Running it only enqueues kernels and copies, which
 * is what lets batches be captured in a CUDA graph.  Replaces, for repeated requests over the
 * same states, the per-call planning of coulombo.cpp:121-151. */
int cl_request_create(cl_ctx* ctx, int64_t n_int, const int16_t* spec, cl_request** out);
/* A prepared request of one shard (see cl_compute_shard): runs write zeros for the other shards'
 * integrals; cl_request_create is shard 0 of 1. */
int cl_request_create_shard(cl_ctx* ctx, int64_t n_int, const int16_t* spec, int shard, int n_shards,
                            cl_request** out);
int cl_request_run(cl_request* req, double* out /* [n_int]{re,im} */);
void cl_request_destroy(cl_request* req);

/* A batch of requests on distinct contexts of one GPU (e.g. nanostructures of uneven grid
 * sizes).  The first cl_batch_run runs each request once, then captures all of them as
 * parallel branches of one CUDA graph (each on its own context's stream); every run launches
 * that graph once.  outs[i] receives request i's values.  No reference counterpart (the
 * reference runs one structure per process). */
int cl_batch_create(cl_request** reqs, int n, cl_batch** out);
int cl_batch_run(cl_batch* batch, double** outs);
/* Device time (ms, CUDA events around the graph launch) of the last cl_batch_run. */
int cl_batch_last_ms(cl_batch* batch, double* ms);
void cl_batch_destroy(cl_batch* batch);

/* ---------------------------------------------------------------------------------------
 * FFT engine (FourierPlan seam, src/FourierPlan.hpp:17-39)
 * ------------------------------------------------------------------------------------- */

/* In-place batched 3D complex FFT of `batch` grids nx*ny*nz (x fastest), sign -1 forward or
 * +1 backward, unnormalised (FFTW's convention).  fp32 != 0 runs the FP32 stages (data are
 * rounded to float on upload and widened back).  Replaces fftw_execute on the plans of
 * src/CoulombCalculator.cpp:17-32. */
int cl_fft3d(int nx, int ny, int nz, int batch, int sign, int fp32, double* data);

/* Allocation-free variant of cl_fft3d for callers that cannot call cudaMalloc (those whose
 * pool or arena owns all device memory, or whose latency-critical path must not let an
 * allocation synchronise the device).  No counterpart in the reference: it exists for this
 * library's callers.  `data` is a DEVICE pointer to batch*nx*ny*nz complex doubles,
 * 16-byte aligned, transformed in place on the legacy default stream; the call returns
 * after the transform has finished.  It allocates nothing: the twiddle tables live in a
 * fixed 192 KiB array inside the library (held by every GPU that loads it until exit), so
 * each axis is limited to 4096 points and longer axes are rejected.  Every call looks up
 * that array's device address on the current device, so a device reset leaves no stale
 * address.  All calls share the array: calls that overlap on the GPU race. */
int cl_fft3d_noalloc(int nx, int ny, int nz, int batch, int sign, double* data);

/* ---------------------------------------------------------------------------------------
 * Host-side helpers (no GPU needed)
 * ------------------------------------------------------------------------------------- */

/* Smallest c * 2^i 3^j 5^k >= n.  Replaces Round::up<2,3,5> (src/Round.hpp:20-49). */
int cl_round_up_235(int n, int c);

/* Lattice-grid detection: per-axis float-GCD step, origin, raw size, 2*3*5 padding, and the
 * cell index of every atom.  pos is [atom][3] in Angstrom; cells may be NULL.
 * Replaces gcd/computeGrid/round4FFT and the cell loop of src/Broadcaster.cpp:8-87, 136-143.
 * Fails with "could not find common grid step" like the reference. */
int cl_detect_grid(const double* pos, int64_t n_atoms, int raw[3], int pad[3],
                   double origin[3], double step[3], int64_t* cells);

/* Number of 1-based (i1..i4) in [1,n_inputs]^4 matching the comma-separated pattern list,
 * and (if specs != NULL and capacity suffices) the matches in lexicographic order as
 * int16[4] each.  Replaces Pattern (src/Pattern.hpp:15-100) and coulombo.cpp:135-148. */
int cl_enumerate_integrals(const char* pattern, int n_inputs, int n_holes, int64_t* count,
                           int16_t* specs, int64_t capacity);

/* Greedy vertex cover of an undirected graph with self-loops (edges as int pairs);
 * in_cover[v] = 0/1.  Replaces Graph::computeVertexCover (src/Graph.hpp:49-91). */
int cl_vertex_cover(int n_vertices, int64_t n_edges, const int32_t* edges, uint8_t* in_cover);

/* The reference's execution plan for a list of integrals: steps[i] = {id, left, lconj,
 * right, rconj} in execution order.  Replaces MasterPlanner (src/Planner.hpp:71-117). */
int cl_plan(int n_inputs, int64_t n_int, const int16_t* spec, int32_t* steps /* [n_int][5] */);

/* Writes the XXXX.txt files of the integrals: one file per electron/hole class that has values,
 * named out_prefix + class + ".txt", rows "%2d %2d %2d %2d   %17.14f %17.14f\n" in (ni, nj, nk,
 * nl) order with the hole numbering reversed.  The lines are formatted on `threads` host threads
 * (<= 0: all) and written in order, byte for byte as the serial loop of the reference.
 * Replaces coulombo.cpp:213-262. */
int cl_write_integrals(const char* out_prefix, int n_holes, int n_electrons, int64_t n_int, const int16_t* spec,
                       const double* values, int threads);

#ifdef __cplusplus
}
#endif

#endif /* COULOMBO_LATTICE_H */
