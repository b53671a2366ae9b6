/* gpuqt.h — the C ABI of the B200 linear-scaling quantum transport library.
 *
 * Plain C types only: pointers, sizes, doubles. Every call returns a gqt_status
 * (0 = success) and never exits the process; gqt_last_error() gives the message of
 * the last failure on the calling thread. The C++ surface in include/lsqt/ (Model,
 * Hamiltonian, Vector, find_* — the reference's own names) is a thin layer over
 * these calls and turns a failure into the reference's print-and-exit.
 *
 * Each entry point names the reference interface it replaces (paths relative to the
 * reference checkout). Device work is issued on the calling thread's current stream
 * (gqt_set_stream); calls that return host data synchronise that stream.
 *
 * Layout on the device (owned by the handles):
 *   vectors      interleaved complex, [site][vector] (double2 or float2)
 *   Hamiltonian  ELL column-major [m*n + i]: int32 neighbour index, double2 hopping,
 *                double xx; double on-site potential [n]; int32 row length [n] only
 *                when rows are ragged; where the entries take at most GQT_MAX_CODES
 *                distinct values, also a one-byte code per entry and the table of
 *                those values (the coded format).
 */
#ifndef GPUQT_H
#define GPUQT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int gqt_status;
enum {
  GQT_OK = 0,
  GQT_ERR_ARG = 1,     /* invalid argument (null handle, size mismatch, bad label) */
  GQT_ERR_CUDA = 2,    /* a CUDA runtime call failed */
  GQT_ERR_ALLOC = 3,   /* device or host allocation failed */
  GQT_ERR_INPUT = 4,   /* malformed input file or model parameters */
  GQT_ERR_IO = 5,      /* a file could not be opened or written */
  GQT_ERR_STATE = 6    /* call not valid in the handle's current state */
};

/* Arithmetic forms of a Hamiltonian/vector pair. */
enum {
  GQT_FP64 = 0, /* plain: FP64 vectors, FP64 operator, reference operation order */
  GQT_FP32 = 1, /* precision: FP32 vectors, FP64 operator and FP64 compensated sums */
  /* No counterpart in the reference. A form of the moment recurrence only (the
   * precision argument of gqt_moments_form / _device_form / gqt_moments_doubled*, on
   * FP64 or FP32 vectors of one model, 1, 4 or 16 per launch): each Chebyshev vector
   * is stored as FP32 plus a BF16 residual (12 bytes per complex element against
   * FP64's 16, about 32 significant bits), with the FP64 operator and FP64 sums.
   * DOS and VAC agree with FP64 to about 1e-8 pointwise, where FP32 storage reaches a
   * few 1e-6 at late VAC times. Vectors of this form cannot be created. */
  GQT_FP32X = 2,
  /* No counterpart in the reference. A form of the moment recurrence only (as
   * GQT_FP32X; 4, 16 or 32 vectors per launch): FP32 vectors and FP32 hoppings (each
   * hopping and potential divided by energy_max in FP64, then held as two FP32 parts,
   * hi = RN(a) and lo = RN(a - hi)), the Chebyshev recurrence in FP32, and the moments
   * summed in FP64 from the stored FP32 values. Runs on GQT_FP32 vectors as they are,
   * or on FP32 copies of GQT_FP64 ones. A realisation batch runs it through the staged
   * step only (coded operator, 16 or 32 vectors, 16 for symmetric sets). */
  GQT_FP32R = 3
};

typedef struct gqt_ham gqt_ham;
typedef struct gqt_vec gqt_vec;

/* ---------------------------------------------------------------- runtime */
const char* gqt_last_error(void);
gqt_status gqt_version(int* major, int* minor);
/* Stream (a cudaStream_t) used by subsequent calls from this thread; NULL = legacy
 * default stream, as the reference uses (src/hamiltonian.cu:228). */
gqt_status gqt_set_stream(void* stream);
void* gqt_get_stream(void);
/* Synchronise the current stream and report any asynchronous kernel error. */
gqt_status gqt_sync(void);
/* Kernel launches this thread has issued since the last reset (all of them are this
 * library's own kernels). */
uint64_t gqt_launch_count(void);
void gqt_reset_launch_count(void);

/* ---------------------------------------------------------------- Hamiltonian */
/* The model's ELL arrays, row-major [i*max_neighbor + m] on the host, exactly as
 * Model holds them (src/model.h:55-60). Entries past neighbor_number[i] are ignored.
 * xx may be NULL when the commutator/current are never applied. */
typedef struct {
  int n;
  int max_neighbor;
  double energy_max;
  const int* neighbor_number;
  const int* neighbor_list;
  const double* potential;
  const double* hopping_real;
  const double* hopping_imag;
  const double* xx;
} gqt_ell_desc;

/* Replaces Hamiltonian::Hamiltonian(Model&) / initialize_gpu
 * (src/hamiltonian.cu:124-131, :27-89): validates every neighbour index on the host
 * (0 <= j < n, row length <= max_neighbor) before anything is uploaded. */
gqt_status gqt_ham_create(const gqt_ell_desc* desc, gqt_ham** out);
/* Replaces Hamiltonian::~Hamiltonian (src/hamiltonian.cu:133-150). */
gqt_status gqt_ham_destroy(gqt_ham* h);
gqt_status gqt_ham_info(const gqt_ham* h, int* n, int* max_neighbor, int* uniform_rows,
                        double* energy_max);

/* Operator storage formats (no counterpart in the reference, whose device layout is
 * GQT_FORMAT_ELL). When the entries (j - i, hopping, xx) of the ELL take at most
 * GQT_MAX_CODES distinct values — lattice models do — gqt_ham_create also builds the
 * coded form: one byte per entry into a table of those values, which the kernels
 * read from shared memory. The arithmetic is unchanged (the same doubles in the same
 * order, so the FP64 form stays bit-identical to the reference); the operator's bytes
 * per site drop from 20 z to z. The coded form is used by default when it exists;
 * gqt_ham_set_format selects a format, gqt_ham_format reports the one in use and the
 * table size (0 when there is no coded form). */
#define GQT_MAX_CODES 256
enum { GQT_FORMAT_ELL = 0, GQT_FORMAT_CODED = 1 };
gqt_status gqt_ham_set_format(gqt_ham* h, int format);
gqt_status gqt_ham_format(const gqt_ham* h, int* format, int* n_codes);

/* Realisation batches (no counterpart in the reference, which runs one model per
 * process): `count` independent models — disorder realisations, lattices of uneven
 * sizes — as one block-diagonal operator, so one launch per Chebyshev step advances
 * all of them and all their vectors. Model r occupies sites
 * [offset_r, offset_r + n_r) of the batch's vectors; each model is padded to a whole
 * number of GQT_BATCH_TILE_SITES sites (padding sites carry zero vectors) and its
 * operator is stored pre-divided by its own energy_max. On a batch, gqt_moments
 * returns moments per model (layout [r][vector][m]); gqt_apply and
 * gqt_kernel_polynomial apply the scaled operator; the evolution and current
 * entry points are rejected (their Bessel coefficients depend on each model's
 * energy_max). */
#define GQT_BATCH_TILE_SITES 1024
#define GQT_MAX_REALISATIONS 32
gqt_status gqt_ham_create_batch(const gqt_ell_desc* descs, int count, gqt_ham** out);
/* The batch step hands out tiles of 256, 512 or 1024 consecutive sites (each divides
 * the padding, so a tile never straddles two models); gqt_autotune_nvec picks the
 * fastest, gqt_ham_set_batch_tile sets one (GQT_ERR_STATE on a single model), and
 * gqt_ham_batch_tile reports the one in use (0 on a single model). Moments agree
 * between tile sizes to rounding (the per-block sums group differently). */
gqt_status gqt_ham_set_batch_tile(gqt_ham* h, int tile_sites);
gqt_status gqt_ham_batch_tile(const gqt_ham* h, int* tile_sites);

/* The moment loop of the FP64 form (no counterpart in the reference, which launches
 * one step at a time). window 0: one launch per Chebyshev step (the default). window
 * S >= 2: the wavefront loop, S steps per persistent launch. The sites are cut into
 * chunks; each block takes (step, chunk) items from a ticket counter in an order in
 * which every item depends only on earlier tickets, and starts one as soon as the
 * previous step is done on the chunks its rows reach. So the S steps run as a wave
 * through L2 and only the leading step reads its vectors from HBM. It applies to one
 * model, one FP64 vector, the coded operator, rows of 3, 4 or 6 entries, and a halo
 * small against the lattice. Other loops run step by step. Every T_m is bit-identical
 * between the two loops; the moments are summed in another fixed order (equal to
 * 1e-12). chunk_sites (a multiple of 256; 0: 1024) sets the chunk: smaller chunks
 * shorten the distance at which the next step reuses a chunk's data, larger ones
 * spend less on each item's hand-over. gqt_ham_loop reports the window and, once a loop has run, the plan (chunks
 * and halo in chunk positions; halo -2: not applicable). */
gqt_status gqt_ham_set_loop(gqt_ham* h, int window, int chunk_sites);
gqt_status gqt_ham_loop(const gqt_ham* h, int* window, int* chunks, int* halo);

/* The staged step of the GQT_FP32 and GQT_FP32R moment loops (no counterpart in the
 * reference) over the coded operator, for 16 or 32 vectors and rows of 3, 4 or 6
 * entries. The sites are cut into tiles; per tile, one thread copies the rows of
 * T_{k-1} its gathers read (a few windows of frequent neighbour offsets, found at
 * upload) and its T_{k-2} rows into shared memory with bulk asynchronous copies,
 * several tiles ahead, and the block computes from shared memory (left is read into
 * registers). Entries whose offset lies in no window (periodic wraps, and the least
 * used windows when two stages of all do not fit) gather from global memory. Every
 * T_m is bit-identical to the unstaged step's; moments agree to FP64 rounding (another
 * summation order).
 * stages: -1 off; 0 automatic (the default), as measured fastest on B200: GQT_FP32R
 * loops are staged, GQT_FP32 loops on rows of 6; 1 every loop, as many stages as fit;
 * 2..4 every loop, that many stages.
 * gqt_ham_staging reports the setting and the windows (lo/hi: room for 8 ints each,
 * or null); windows 0 means the step is never staged for this operator. */
gqt_status gqt_ham_set_staging(gqt_ham* h, int stages);
gqt_status gqt_ham_staging(const gqt_ham* h, int* stages, int* windows, int* lo, int* hi);
/* The stages and windows the staged step would use in a moment loop of nvec vectors in
 * `precision` (GQT_FP32 or GQT_FP32R; symmetric != 0: the loop of symmetric moment
 * sets) under the current setting; *stages = 0 when that loop is not staged. No
 * counterpart in the reference. */
gqt_status gqt_ham_stage_plan(const gqt_ham* h, int nvec, int precision, int symmetric,
                              int* stages, int* windows);
gqt_status gqt_ham_realisations(const gqt_ham* h, int* count);
gqt_status gqt_ham_realisation(const gqt_ham* h, int r, int* offset, int* n,
                               double* energy_max);
/* Project autotuner for the batched moment loop: times n_moments Chebyshev steps for
 * each candidate number of vectors per launch (a supported nvec of `precision`) on
 * this Hamiltonian and returns the one with the highest site-moments/s in *best
 * (rates[k] receives candidate k's best rate; may be NULL). For every candidate it
 * also picks the vector-block shape of the step (vectors per thread, FP32: 4 or 2)
 * and, on a realisation batch, the tile size (256, 512 or 1024 sites), keeping the
 * fastest for later launches. GQT_FP32R is probed on FP32 vectors with its own staged
 * tiles (on a batch its candidates are 16 and 32). Allocates and frees its own probe
 * vectors. */
gqt_status gqt_autotune_nvec(const gqt_ham* h, int precision, int n_moments,
                             const int* candidates, int n_candidates, int* best,
                             double* rates);

/* ---------------------------------------------------------------- vectors */
/* Replaces Vector::Vector(int) (src/vector.cu:61-70): nvec vectors of n sites,
 * zero-initialised. precision is GQT_FP64 or GQT_FP32. */
gqt_status gqt_vec_create(int n, int nvec, int precision, gqt_vec** out);
/* Replaces Vector::Vector(Vector&) (src/vector.cu:92-105): deep copy. */
gqt_status gqt_vec_clone(const gqt_vec* src, gqt_vec** out);
/* Replaces Vector::~Vector (src/vector.cu:107-116). */
gqt_status gqt_vec_destroy(gqt_vec* v);
gqt_status gqt_vec_info(const gqt_vec* v, int* n, int* nvec, int* precision);
/* Device address of the interleaved data ([site][vector] complex). */
void* gqt_vec_data(gqt_vec* v);
/* Replaces Vector::copy_from_host (src/vector.cu:199-208): split real/imag host
 * arrays of n*nvec doubles, vector-major (vector k occupies [k*n, (k+1)*n)). */
gqt_status gqt_vec_upload(gqt_vec* v, const double* real_part, const double* imag_part);
/* Replaces Vector::copy_to_host (src/vector.cu:210-219). */
gqt_status gqt_vec_download(const gqt_vec* v, double* real_part, double* imag_part);
/* Replaces Vector::copy (src/vector.cu:140-148): dst = src. */
gqt_status gqt_vec_copy(gqt_vec* dst, const gqt_vec* src);
/* Replaces Vector::add (src/vector.cu:129-137): dst += src. */
gqt_status gqt_vec_add(gqt_vec* dst, const gqt_vec* src);
/* Replaces Vector::apply_sz (src/vector.cu:175-183): dst = S_z src (sign flips on odd
 * sites). */
gqt_status gqt_vec_apply_sz(gqt_vec* dst, const gqt_vec* src);
/* Replaces Vector::swap (src/vector.cu:221-228): exchanges the device buffers. */
gqt_status gqt_vec_swap(gqt_vec* a, gqt_vec* b);
gqt_status gqt_vec_zero(gqt_vec* v);

/* ---------------------------------------------------------------- operators */
/* Replaces Hamiltonian::apply (src/hamiltonian.cu:225-237): out = H in / E_max. */
gqt_status gqt_apply(const gqt_ham* h, const gqt_vec* in, gqt_vec* out);
/* Replaces Hamiltonian::apply_commutator (:308-320): out = [X,H] in / E_max. */
gqt_status gqt_apply_commutator(const gqt_ham* h, const gqt_vec* in, gqt_vec* out);
/* Replaces Hamiltonian::apply_current (:387-399): out = V in (unscaled). */
gqt_status gqt_apply_current(const gqt_ham* h, const gqt_vec* in, gqt_vec* out);
/* Replaces Hamiltonian::kernel_polynomial (:970-984): s2 = 2 H s1 / E_max - s0.
 * s2 may alias s0 (each site reads its s0 value before writing s2). */
gqt_status gqt_kernel_polynomial(const gqt_ham* h, const gqt_vec* s0, const gqt_vec* s1,
                                 gqt_vec* s2);
/* Replaces Hamiltonian::chebyshev_01 (:447-460). */
gqt_status gqt_chebyshev_01(const gqt_ham* h, const gqt_vec* s0, const gqt_vec* s1,
                            gqt_vec* out, double bessel_0, double bessel_1, int direction);
/* Replaces Hamiltonian::chebyshev_2 (:599-614); label 1..4 as in the reference. */
gqt_status gqt_chebyshev_2(const gqt_ham* h, const gqt_vec* s0, const gqt_vec* s1,
                           gqt_vec* s2, gqt_vec* out, double bessel_m, int label);
/* Replaces Hamiltonian::chebyshev_1x (:652-662). */
gqt_status gqt_chebyshev_1x(const gqt_ham* h, const gqt_vec* in, gqt_vec* out,
                            double bessel_1);
/* Replaces Hamiltonian::chebyshev_2x (:856-882). */
gqt_status gqt_chebyshev_2x(const gqt_ham* h, const gqt_vec* s0, const gqt_vec* s0x,
                            const gqt_vec* s1, const gqt_vec* s1x, gqt_vec* s2,
                            gqt_vec* s2x, gqt_vec* out, double bessel_m, int label);

/* ---------------------------------------------------------------- reductions */
/* Replaces Vector::inner_product_1 + inner_product_2 (src/vector.cu:331-344,
 * :425-436) for one moment: <left|state> per vector, FP64 compensated sums.
 * re/im hold nvec values. */
gqt_status gqt_inner_product(const gqt_vec* state, const gqt_vec* left, double* re,
                             double* im);

/* Stage 1 of the reference's two-stage reduction (Vector::inner_product_1,
 * src/vector.cu:331-344): <left|state> (nvec = 1) written to element `index` of the
 * FP64 vector `target` on the device, without synchronising. */
gqt_status gqt_inner_product_into(const gqt_vec* state, const gqt_vec* left, gqt_vec* target,
                                  int index);
/* Stage 2 (Vector::inner_product_2, src/vector.cu:425-436): out[m] = sum of
 * in[m*segment .. m*segment+segment-1] for m < count; FP64 vectors, nvec = 1. */
gqt_status gqt_vec_segment_sum(const gqt_vec* in, int segment, int count, gqt_vec* out);

/* ---------------------------------------------------------------- algorithms */
/* Replaces find_moments_chebyshev (src/sigma.cu:33-61):
 * mu_m = <left| T_m(H/E_max) |right>, m = 0..n_moments-1, for each of the nvec
 * vectors. mu_re/mu_im are host arrays of nvec*n_moments doubles, vector-major.
 * The Chebyshev step and the moment partial sums run in one fused kernel per
 * moment; the n_moments launches are replayed from a CUDA graph. */
gqt_status gqt_moments(const gqt_ham* h, const gqt_vec* left, const gqt_vec* right,
                       int n_moments, double* mu_re, double* mu_im);
/* As gqt_moments, but leaves the moments on the device (mu_dev: nvec*n_moments
 * double2 (re, im), moment-major [m*nvec + k]; for a realisation batch
 * [m][r][k], n_moments*count*nvec entries) and does not synchronise. */
gqt_status gqt_moments_device(const gqt_ham* h, const gqt_vec* left, const gqt_vec* right,
                              int n_moments, void* mu_dev);
/* As gqt_moments / gqt_moments_device, with the Chebyshev recurrence run in the
 * arithmetic form `precision` whatever the form of left and right: FP64 states (for
 * instance time-evolved ones, which keep their full precision across evolution
 * steps) converted once into FP32 workspace vectors for the FP32-storage moment
 * loop. With precision equal to the vectors' form this is gqt_moments. */
gqt_status gqt_moments_form(const gqt_ham* h, const gqt_vec* left, const gqt_vec* right,
                            int n_moments, int precision, double* mu_re, double* mu_im);
gqt_status gqt_moments_device_form(const gqt_ham* h, const gqt_vec* left,
                                   const gqt_vec* right, int n_moments, int precision,
                                   void* mu_dev);
/* The symmetric moment set mu_m = <phi|T_m(H~)|phi>, m < n_moments, from n_moments / 2
 * Chebyshev steps, by T_j T_k = (T_{j+k} + T_{|j-k|}) / 2 (KPM "doubling": each step
 * fuses <T_k|T_k> and <T_{k-1}|T_k>; mu_2k = 2 <T_k|T_k> - mu_0, mu_{2k-1} =
 * 2 <T_{k-1}|T_k> - mu_1). No counterpart in the reference, whose loop takes n_moments
 * steps (find_moments_chebyshev, src/sigma.cu:33-61, with left = right): same moments
 * up to rounding of order 1e-15 mu_0 per moment in the FP64 form, not bit for bit.
 * precision as in gqt_moments_form; the operator must be Hermitian (checked at upload,
 * GQT_ERR_STATE otherwise); at most 16 vectors, 32 for a realisation batch (moments
 * per realisation, as gqt_moments).
 * Outputs as gqt_moments (host) / gqt_moments_device (device, [m][vector] double2). */
gqt_status gqt_moments_doubled(const gqt_ham* h, const gqt_vec* state, int n_moments,
                               int precision, double* mu_re, double* mu_im);
gqt_status gqt_moments_doubled_device(const gqt_ham* h, const gqt_vec* state, int n_moments,
                                      int precision, void* mu_dev);
/* dst = src across forms (FP64 <-> FP32, same sites and vector count); rounds to
 * nearest when narrowing. */
gqt_status gqt_vec_convert(gqt_vec* dst, const gqt_vec* src);
/* Replaces evolve (src/sigma.cu:116-151): state <- U(direction * dt) state with
 * dt_scaled = dt * E_max. The Bessel coefficients J_m(dt_scaled) come from the host
 * libm (j0/j1/jn) and the series stops at the first m >= 2 with |J_m| < 1e-15, as
 * the reference does. */
gqt_status gqt_evolve(const gqt_ham* h, int direction, double dt_scaled, gqt_vec* state);
/* Replaces evolvex (src/sigma.cu:157-200): state <- [X, U(dt)] state (direction +1)
 * or [U(-dt), X] state (direction -1). */
gqt_status gqt_evolvex(const gqt_ham* h, int direction, double dt_scaled, gqt_vec* state);

/* Replaces apply_damping + perform_chebyshev_summation (src/sigma.cu:76-110): the
 * Jackson-damped Chebyshev sum of the real parts of mu at each energy (host work).
 * mu_re/mu_im are damped in place, as the reference does. */
gqt_status gqt_chebyshev_summation(int n_moments, double* mu_re, double* mu_im,
                                   int n_energy, const double* energy, double energy_max,
                                   double volume, double* out);

/* ---------------------------------------------------------------- model and driver */
typedef struct gqt_model gqt_model;
/* Replaces Model::Model(std::string) (src/model.cu:30-65): reads para.in and the
 * lattice or general-model files of input_dir, builds the ELL arrays and draws the
 * disorder on the reference's single std::mt19937 stream (seed 12345678, as the
 * reference's DEBUG build; the optional para.in keywords `seed`, `disorder_seed` and
 * `phase_seed` override it). Diagnostics go to stdout as the reference prints them
 * when verbose is nonzero. */
gqt_status gqt_model_load(const char* input_dir, int verbose, gqt_model** out);
gqt_status gqt_model_destroy(gqt_model* m);
/* The model's ELL arrays (host memory owned by the model, valid until destroy). */
gqt_status gqt_model_ell(const gqt_model* m, gqt_ell_desc* desc);
/* Scalar parameters: number_of_moments, number_of_energy_points,
 * number_of_steps_correlation, number_of_random_vectors, and volume. */
gqt_status gqt_model_params(const gqt_model* m, int* n_moments, int* n_energy, int* n_steps,
                            int* n_random_vectors, double* volume);
gqt_status gqt_model_energy(const gqt_model* m, double* energy);
gqt_status gqt_model_time_step(const gqt_model* m, double* time_step);
/* Replaces Model::initialize_state (src/model.cu:77-109): the next random-phase
 * vector (orbital < 0) or the local-orbital vector sqrt(N) e_orbital, drawn on the
 * model's generator; re/im are n host doubles. */
gqt_status gqt_model_initial_state(gqt_model* m, int orbital, double* re, double* im);
/* Replaces lsqt(std::string) (src/lsqt.cu:135-152): the full run for one input
 * directory, appending dos.out / vac0.out / vac.out / msd.out / S.out / ldos.out
 * with the reference's formats. precision selects the arithmetic form of the moment
 * recurrence (GQT_FP64, GQT_FP32, or GQT_FP32R, which needs batch_vectors 4 or 16, a
 * number of random vectors divisible by 4 and no local orbitals); states and their
 * time evolution stay FP64. */
gqt_status gqt_lsqt(const char* input_dir, int precision, int verbose);
/* gqt_lsqt with checkpoint / resume; no counterpart in the reference. A checkpoint
 * (input_dir/lsqt.checkpoint: the next row's position, the generator state, the
 * evolved states and the output file sizes) is resumed when present and written
 * every `checkpoint_every` rows (para.in) and, when max_rows > 0, after max_rows
 * rows, where the call stops with *finished = 0. A completed run removes the
 * checkpoint and sets *finished = 1. A resumed run truncates rows written after its
 * checkpoint and writes the same bytes as an uninterrupted run. With max_rows <= 0
 * and no checkpoint_every this is gqt_lsqt. para.in `output_moments` also appends
 * each row's raw moments to <name>_moments.bin (16-byte header "GQTMOMv1",
 * int32 number_of_moments, int32 0; then per row number_of_moments (re, im) doubles,
 * little-endian). */
gqt_status gqt_lsqt_run(const char* input_dir, int precision, int verbose, long long max_rows,
                        int* finished);

/* ---------------------------------------------------------------- no-allocation step */
/* No counterpart in the reference. One fused Chebyshev step with its moment, the
 * kernel that gqt_moments repeats, for callers that drive the recurrence themselves
 * and cannot let the library allocate device memory: a host that has already handed
 * all of HBM to its own pool (a lattice sized to fill the GPU, or a framework's
 * caching allocator) gets no memory from cudaMalloc, and in a loop that is being
 * timed or captured, cudaMalloc's implicit device-wide synchronisation is not
 * allowed either. This call allocates nothing: the block partials and the arrival
 * counter of the moment reduction live in a static device array of
 * GQT_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until exit.
 *
 *   mode 0: out = H t1 / E_max           (t0 ignored; the first step)
 *   mode 1: out = 2 H t1 / E_max - t0    (out may alias t0; never t1 or left)
 *   mu_dev: device array of nvec double2 receiving <left|out> (re, im)
 *
 * FP64 vectors only (the reference's arithmetic; out is bit-identical to
 * gqt_apply / gqt_kernel_polynomial), the operator read in the Hamiltonian's current
 * format (gqt_ham_set_format; the coded table goes to shared memory, no allocation).
 * The launch uses at most
 * GQT_NOALLOC_SCRATCH_BYTES / (32 * nvec) blocks; a call whose reduction would need
 * more scratch than that is rejected with GQT_ERR_ARG. The first call on a device
 * looks up the array's device address (cudaGetSymbolAddress) and must come before
 * any stream capture on that device. All calls share the one array: calls whose
 * kernels can overlap on the GPU (different streams or threads, without ordering
 * between them) race on it and must not be issued. */
#define GQT_NOALLOC_SCRATCH_BYTES (1u << 20)
gqt_status gqt_chebyshev_step_noalloc(const gqt_ham* h, int mode, const gqt_vec* t0,
                                      const gqt_vec* t1, gqt_vec* out, const gqt_vec* left,
                                      void* mu_dev);

#ifdef __cplusplus
}
#endif
#endif
