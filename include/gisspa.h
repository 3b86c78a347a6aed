/*
 * gisspa.h -- C ABI of the B200-native GisSPA template-matching search.
 *
 * The reference (Autumn1998/GisSPA) has no library interface: its boundary is
 * the `./main <config>` process, and its search lives in host functions that
 * take raw cufftComplex device buffers (main.cu).  Each entry point below
 * replaces one of those host stages; the comment names the reference code it
 * stands in for.  The drop-in CLI (gisspa_main, csrc/driver) and the Python
 * wrapper (gisspa_b200/__init__.py) call only these functions.
 *
 * Conventions
 *  - Every function returns an int status (GS_OK == 0).  Nothing calls exit().
 *  - Pointers named host_* are host memory owned by the caller; the context
 *    owns all device memory it allocates.  *_device entry points take device
 *    pointers on the context's device.
 *  - One context per host thread; a context runs its work on its own CUDA
 *    stream and calls on one context must not overlap.
 *  - Angles are degrees, defocus values micrometres exactly as written in the
 *    reference's input list (positive = underfocus).
 */
#ifndef GISSPA_H
#define GISSPA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The reference prints and exit(-1)s on every failure
 * (GPU_func.cuh:33-41); here each failure is returned to the caller. */
#define GS_OK 0
#define GS_ERR_ARG 1         /* bad argument (null pointer, size, geometry) */
#define GS_ERR_OOM 2         /* device or host allocation failed */
#define GS_ERR_CUDA 3        /* a CUDA runtime call or kernel failed */
#define GS_ERR_STATE 4       /* call out of order (e.g. search before templates) */
#define GS_ERR_UNSUPPORTED 5 /* valid input outside what this build handles */
#define GS_ERR_TIMEOUT 6     /* a bounded device wait gave up */
#define GS_ERR_IO 7          /* file could not be read or written */

/* Search parameters: the numeric fields of the reference's
 * struct Parameters (EMReader/DataReader.h:14-42), same meaning and defaults
 * (see gs_params_default). */
typedef struct gs_params {
    float apix;        /* angpix: pixel size, A */
    float phi_step;    /* phistep: in-plane angle step, deg */
    float kk;          /* kk: overlapping density parameter */
    float energy;      /* energy: kV */
    float cs;          /* cs: spherical aberration, mm */
    float highres;     /* Highres: high-resolution cut, A */
    float lowres;      /* Lowres: low-resolution cut, A */
    float d_m;         /* diameter: particle diameter, px */
    float thres;       /* threshold: score threshold (default 7) */
    int window_size;   /* window_size: window l (default 320) */
    int overlap;       /* overlap between windows, px (default -1) */
    int phase_flip;    /* phase_flip 0/1 (default 0) */
    int norm_type;     /* norm_type: 0 = peak / sigma per map, 1 = per-pixel
                          z-score over all templates and angles (default 0) */
    int invert;        /* invert 0/1 (default 0) */
    float ampconst;    /* amplitude contrast (fixed 0.07 in the reference) */
    float a, b, b2;    /* noise-curve constants (DataReader.h:25) */
    float bfactor, bfactor2, bfactor3; /* signal-curve constants */
    int precision;     /* arithmetic of the correlation's DFT stages (no
                          reference counterpart; default GS_PREC_FP32) */
} gs_params;

/* GS_PREC_FP32: every FFT stage in FP32 on the CUDA cores (the reference's
 * precision).  GS_PREC_TC_BF16 / GS_PREC_TC_FP16: the N2-point DFT stage of
 * the correlation (window l = 16 * N2 with N2 = 32, 45 or 48, persistent
 * path) runs on the tensor cores as a GEMM with operands split into 16-bit
 * (hi, lo) parts, hi*hi + lo*hi + hi*lo accumulated in FP32; other stages
 * stay FP32.  Other windows, the two-pass path and norm_type 1 return
 * GS_ERR_UNSUPPORTED with these modes; GS_PREC_TC_FP16 also needs
 * phase_flip 1 (its data operand relies on amplitude-normalised spectra to
 * stay inside the FP16 range). */
#define GS_PREC_FP32 0
#define GS_PREC_TC_BF16 1
#define GS_PREC_TC_FP16 2
/* GS_PREC_TC_FULL / GS_PREC_TC_FULL_1P (window 720, persistent path,
 * norm_type 0): every DFT stage of the correlation (16- and 45-point, both
 * passes) runs on the tensor cores with FP16 operands and FP32 accumulation,
 * the data rounded to FP16 once per stage and the DFT matrix split into
 * (hi, lo) FP16 parts (two products) or rounded once (_1P, one product); each
 * unit's spectrum is scaled by a power of two to stay inside the FP16 range
 * and the row-pass maps are kept in FP16.  Scores stay within 1e-3 relative
 * of the FP64 oracle (a few 1e-4 measured); other windows return
 * GS_ERR_UNSUPPORTED. */
#define GS_PREC_TC_FULL 3
#define GS_PREC_TC_FULL_1P 4

/* Per-micrograph CTF line values as in the input list
 * (DataReader.cpp:366-388: defocus=, dfdiff=, dfang=). */
typedef struct gs_ctf {
    float defocus; /* um, positive underfocus */
    float dfdiff;  /* um */
    float dfang;   /* deg */
} gs_ctf;

/* One output line of the reference's writeScoreToDisk (main.cu:974-989). */
typedef struct gs_pick {
    int angle_index;   /* index in the in-plane angle loop */
    float phi;         /* third Euler angle as printed: 360 - euler3, wrapped */
    int window_x;      /* window column i */
    int window_y;      /* window row j */
    int template_index;/* J (row of the Euler file) */
    float center_x;    /* micrograph pixel x of the peak */
    float center_y;
    float score;       /* peak / sigma-without-peak */
} gs_pick;

/* Per (angle, window, template) result of the last search, dense. */
typedef struct gs_unit {
    float score;  /* NaN when the map had zero variance (no pick possible) */
    int pos;      /* argmax flat index y*l + x in window coordinates */
    float peak;   /* max(0, border-masked max) */
    float sigma;  /* std of the map without the peak */
} gs_unit;

/* Search geometry derived from the parameters, templates and micrograph. */
typedef struct gs_geometry {
    int l;          /* window size after the template-size adjustment */
    int n_windows_x;
    int n_windows_y;
    int n_angles;
    int n_templates;
} gs_geometry;

const char* gs_status_string(int status);
int gs_version(void);

/* Reference defaults of struct Parameters (DataReader.h:16-42); required
 * keys are set to -1 like the reference's "not given" marker. */
int gs_params_default(gs_params* p);

/* Context on one CUDA device; replaces main.cu:1071 cudaSetDevice + the
 * stream of main.cu:274.  Owns a stream and all device buffers.  Opaque to
 * callers: declared here so that C and C++ callers name one type. */
struct gs_ctx;
typedef struct gs_ctx gs_ctx;
int gs_ctx_create(int device, struct gs_ctx** out);
int gs_ctx_destroy(struct gs_ctx* ctx);
/* Last error text of this context ("" if none). */
const char* gs_ctx_last_error(struct gs_ctx* ctx);

/* Template preprocessing, once per run.  Replaces readAndPaddingTemplate +
 * edgeNormalize + handleTemplate (main.cu:182-474): pad to l x l, edge-ring
 * normalise, whiten by radial shells, band-pass and |CTF| x Wiener weight with
 * `first_ctf` (the reference weights every template with the FIRST
 * micrograph's CTF, main.cu:1106), amplitude-normalise, inverse FFT.
 * host_templates: n x ty x tx float32, row-major. */
int gs_set_templates(struct gs_ctx* ctx, const gs_params* p, const float* host_templates,
                     int n, int tx, int ty, const gs_ctf* first_ctf);

/* Geometry of a search of an nx x ny micrograph with the loaded templates. */
int gs_get_geometry(struct gs_ctx* ctx, int nx, int ny, gs_geometry* out);

/* One micrograph.  Replaces init_d_image + split_normalize_image +
 * fft_on_img + the angle loop of rotateTemplate and pickPartcles_IMG_NORM
 * (main.cu:523-894, 1230-1257) for norm_type 0, and compute_CCG_sum +
 * compute_CCG_mean + pickPartcles_CCG_NORM (main.cu:718-821, 1170-1229) for
 * norm_type 1.  Picks come back in the reference's line order (angle,
 * window row, window column, template; for norm_type 1 then the 1024-element
 * block of the map); *picks is allocated by the library, release it with
 * gs_picks_free.  norm_type 1 needs window * window to be a multiple of 1024
 * (checked by gs_set_templates: GS_ERR_UNSUPPORTED).
 * host_micrograph: ny x nx float32 row-major. */
int gs_search(struct gs_ctx* ctx, const float* host_micrograph, int nx, int ny,
              const gs_ctf* ctf, gs_pick** picks, size_t* n_picks);

/* Several micrographs, possibly of different sizes, in one search with the
 * loaded templates (no reference counterpart: the reference loops over its
 * input list, main.cu:1149-1269, and re-does every angle's template spectra
 * per micrograph).  All micrographs' windows share the window-spectrum array
 * and each angle's template spectra; the persistent correlation runs over
 * every (window, template pair) of the batch in one launch per angle.  Picks
 * equal those of one gs_search per micrograph; they come back concatenated in
 * micrograph order, picks_per_micrograph[m] (caller array of n_micrographs)
 * telling how many belong to each.  host_micrographs[m]: ny[m] x nx[m]
 * float32 row-major; ctfs[m] its CTF line.  With norm_type 1 the micrographs
 * are searched one after the other. */
int gs_search_batch(struct gs_ctx* ctx, int n_micrographs, const float* const* host_micrographs,
                    const int* nx, const int* ny, const gs_ctf* ctfs, gs_pick** picks, size_t* n_picks,
                    size_t* picks_per_micrograph);

/* Same search with the micrograph already in device memory (ny x nx float32
 * on the context's device).  The micrograph is not modified. */
int gs_search_device(struct gs_ctx* ctx, const float* device_micrograph, int nx, int ny,
                     const gs_ctf* ctf, gs_pick** picks, size_t* n_picks);

/* Copy the dense per-unit table of the last search (n_angles x n_windows x
 * n_templates, that order) into host memory; cap is the element capacity.
 * Only a norm_type 0 search produces it (GS_ERR_STATE otherwise). */
int gs_get_units(struct gs_ctx* ctx, gs_unit* host_out, size_t cap, size_t* n_out);

/* Per-pixel maximum of the normalised correlation over (template, in-plane
 * angle) for micrograph `micrograph` (0-based, in the order given) of the
 * last norm_type 0 search.  No reference counterpart: the reference keeps
 * one peak per (angle, window, template) map (main.cu:856-891), and the
 * picks keep that rule; this map is an additional output.  Each map value
 * is cc / sigma, sigma being that map's standard deviation without its peak
 * as in the score (main.cu:869-876), so at a map's peak pixel it equals the
 * unit's score.  Map pixel (X, Y) (fftshifted window index, as the picks'
 * positions) lands on micrograph pixel (offx + X, offy + Y); the border the
 * score's maximum leaves out (d_m / 4, GPU_func.cu:681) is left out here
 * too, and overlapping windows merge by maximum.  Host outputs, nx * ny
 * each, row-major: value (0 where no map reaches `thres`), template_index and
 * angle_index (-1 there; either may be NULL).  Among equal values the
 * smallest (angle, template) wins.  Only units whose score reaches `thres`
 * are recomputed (no other unit can have a pixel at or above it), with the
 * FP32 kernels whatever the search's precision; a low threshold costs up to
 * a second search. */
int gs_get_pixel_max(struct gs_ctx* ctx, int micrograph, float thres, float* value, int* template_index,
                     int* angle_index);

void gs_picks_free(gs_pick* picks);

/* Timings of the last search, measured with CUDA events on the context's
 * stream (no reference counterpart; the reference prints whole seconds,
 * main.cu:1271-1272).  Fills min(n, GS_TIMING_COUNT) entries:
 *  [0] micrograph preprocessing ms   [1] template spectra ms (all angles)
 *  [2] correlation ms (all angles)    [3] total ms
 *  [4] row-pass kernel ms (sum)       [5] row-pass launches
 *  [6] column-pass kernel ms (sum)    [7] column-pass launches
 * With the persistent correlation kernel, [4]/[5] hold its time and launches
 * (one launch covers gs_get_tuning's [5] angles, the last launch the
 * remainder) and [6]/[7] are zero.  Entries 4-7 are filled only while per-kernel timing
 * is enabled. */
#define GS_TIMING_COUNT 8
int gs_get_timings(struct gs_ctx* ctx, float* out, int n);

/* ---- Off-grid refinement (no reference counterpart) ----
 * The objective of a pick continues the search's score off its grid: the
 * template is re-weighted with the pick's CTF (defocus, dfdiff, dfang of the
 * band-pass x |CTF| Wiener weight, main.cu:434-463), rotated by the pick's
 * angle (the search's bilinear rotation, mask and normalisation,
 * main.cu:669-716), and correlated with the window at the map position pos
 * moved by (dx, dy) pixels (band-limited, through the window spectrum); the
 * score is that correlation over the map's standard deviation (Parseval).
 * At the grid angle, dx = dy = 0 and the CTF of the first micrograph it is the
 * search's score up to the peak's own share of sigma (about 1e-4 relative).
 * Picks refer to the window spectra of the last norm_type 0 search on this
 * context (window: index in its window order, all micrographs of a batch in
 * order; pos: the unit's peak position as gs_get_units reports it). */
typedef struct gs_refine_pick {
    int window;
    int template_index;
    int pos;               /* Y * l + X, map position of the peak */
    float angle;           /* in-plane angle, degrees */
    float dx, dy;          /* sub-pixel shift, pixels */
    float defocus, dfdiff, dfang;  /* um (positive underfocus), um, degrees */
} gs_refine_pick;

typedef struct gs_refine_result {
    float score;
    float d_angle, d_dx, d_dy, d_defocus, d_dfdiff, d_dfang;  /* d score / d parameter */
} gs_refine_result;

/* Objective of n picks and, with with_gradient, its gradient by the adjoint
 * (the forward's spectra are kept on the device for the backward of the same
 * call; nothing is stored across calls).  template_gradients: null, or host
 * memory of n x l x l floats receiving d score / d template base pixels (the
 * whitened template before the CTF weight, l x l). */
int gs_score_grad(struct gs_ctx* ctx, const gs_refine_pick* picks, int n, int with_gradient,
                  gs_refine_result* out, float* template_gradients);

/* `steps` steps of gradient ascent on every pick's objective (angle, shift,
 * defocus, dfdiff, dfang); a step that lowers a pick's score is undone and
 * that pick's step length halved.  picks are updated in place; out receives
 * the final scores and gradients. */
int gs_refine(struct gs_ctx* ctx, gs_refine_pick* picks, int n, int steps, gs_refine_result* out);

/* ---- Duplicate merging of picks ----
 * Replaces python_scripts/remove_repeat_particles_from_list.py: picks are
 * grouped in runs of equal `group` (the script's runs of one micrograph
 * path); inside a run, in order, two picks whose centres are closer than
 * `center` pixels and whose orientations (alt, az, phi, degrees) are closer
 * than `euler_thres` degrees (or than that modulo 180) are duplicates, and
 * the lower score is removed (equal scores remove the earlier pick); a pick
 * already removed when its turn comes is skipped.  keep[k] receives 1 for
 * the picks that stay.  Pair tests run on `device` in FP64, the removal sweep
 * on the host.  Needs no context. */
typedef struct gs_merge_item {
    double x, y;            /* centre, pixels */
    double alt, az, phi;    /* orientation, degrees */
    double score;
    long long group;        /* run id (e.g. micrograph) */
} gs_merge_item;

int gs_merge_duplicates(int device, const gs_merge_item* items, size_t n, double center,
                        double euler_thres, unsigned char* keep);

/* Scheduling the last search used for the persistent correlation (after
 * autotuning when GS_OPT_AUTOTUNE is on): the first min(n, 6) of {ring
 * slots, lag, window block, CTAs per SM (0 = as many as fit), tile width,
 * in-plane angles per launch}. */
int gs_get_tuning(struct gs_ctx* ctx, int* out, int n);

/* Enable (1) or disable (0) per-kernel event timing of the correlation
 * passes; it adds two events per launch. */
int gs_set_kernel_timing(struct gs_ctx* ctx, int enable);

/* Tuning / cross-check options (no reference counterpart).
 * GS_OPT_GENERIC_FFT: 1 = always use the generic mixed-radix kernels, 0 =
 * use the specialised l = 16*N2 kernels where they exist (default). */
#define GS_OPT_GENERIC_FFT 1
/* GS_OPT_TWO_PASS: 1 = run the correlation as separate row and column
 * launches per window, 0 = one persistent launch per angle where the
 * specialised kernels exist (default). */
#define GS_OPT_TWO_PASS 2
/* GS_OPT_WINDOW_BLOCK: windows per block of the persistent launch's unit
 * order (reuse of window and pair spectra in L2); default 4 (8 for the FP32
 * kernel at window 512). */
#define GS_OPT_WINDOW_BLOCK 3
/* GS_OPT_CORR_SLOTS / GS_OPT_CORR_LAG: scratch maps in the persistent
 * launch's ring (default 16) and how many units after its row tiles a unit's
 * column tiles are queued (default 6); slots must exceed lag.  The FP32
 * kernel at window 512 defaults to 32 slots and a lag of 10.  The
 * all-tensor-core modes keep more items in flight and default to 24 slots and
 * a lag of 12 unless either option was set; they need lag >= 1 and
 * slots >= lag + 2 (GS_ERR_UNSUPPORTED otherwise). */
#define GS_OPT_CORR_SLOTS 4
#define GS_OPT_CORR_LAG 5
/* GS_OPT_CORR_CTAS: resident CTAs per SM of the persistent launch (0 = as
 * many as shared memory, registers and TMEM allow; default 0). */
#define GS_OPT_CORR_CTAS 6
/* GS_OPT_GRAPH: 1 = capture the whole angle loop (template spectra +
 * correlation of every angle) as one CUDA graph and launch it once; per-angle
 * timings are then not available (gs_get_timings [1] is 0 and [2] holds the
 * graph's time). */
#define GS_OPT_GRAPH 7
/* GS_OPT_AUTOTUNE: 1 = before the first search of a given (window,
 * templates, windows, precision), time candidate ring slots, lag, window
 * block, CTAs per SM and tile width on angle 0 over up to 8192 units and
 * keep the fastest for this context (gs_get_tuning shows the choice). */
#define GS_OPT_AUTOTUNE 8
/* GS_OPT_CORR_TILE: vectors per tile of the FP32 persistent kernel: 16
 * (256-thread CTAs, two per SM; default) or 8 (128-thread CTAs, four per
 * SM; default at window 512).  The autotuner also tries both. */
#define GS_OPT_CORR_TILE 9
/* GS_OPT_ANGLES_PER_LAUNCH: in-plane angles whose units one persistent
 * correlation launch covers (their pair spectra are computed first, all
 * resident at once).  0 (default) = enough angles for about 16384 (window,
 * template pair) units per launch, with the pair spectra of one launch
 * within 8 GiB; with GS_OPT_AUTOTUNE on, the autotuner then also times 1,
 * a quarter, half and all of that count and keeps the fastest per angle.
 * A count above the angle count is clamped, and so is one whose item
 * indices would overflow. */
#define GS_OPT_ANGLES_PER_LAUNCH 10
int gs_set_option(struct gs_ctx* ctx, int option, int value);

/* Counters of this context since creation (no reference counterpart; the
 * reference reports only its wall time, main.cu:1271-1272). */
typedef struct gs_stats {
    unsigned long long kernel_launches; /* kernels this library launched */
    unsigned long long searches;        /* completed gs_search* calls */
    unsigned long long units;           /* (angle, window, template) units scored */
} gs_stats;
int gs_get_stats(struct gs_ctx* ctx, gs_stats* out);

/* EMAN HDF5 input (host only; needs no GPU and no context).  Replaces the
 * reference's HDF5 branch of emdata::readImage (EMReader/emdata_.cpp:174-199)
 * with libhdf5 behind it: EMhdf (old style, EMReader/emhdf_.cpp:95-265,
 * chosen when the root group has a num_dataset attribute; image `index` is the
 * root dataset named by the index, nx / ny / nz = dims[0] / dims[1] / dims[2]
 * of its dataspace, floating-point data only, equal spacing_row / spacing_col /
 * spacing_sec required) and EMhdf2 (EMAN2 style, EMReader/emhdf2_.cpp:245-362:
 * dataset /MDF/images/<index>/image sized by the EMAN.nx / EMAN.ny / EMAN.nz
 * attributes of its group, integer or float data converted to float).  A
 * negative index reads image 0.  The file must start with the HDF5 signature
 * (EMhdf::is_valid).  On success *host_data holds nx * ny * nz floats, x
 * fastest, to be released with gs_host_free.  Where the reference falls back
 * to a 10 x 10 zero image (missing image, no size attributes, anisotropic
 * spacing, size mismatch) this returns GS_ERR_IO with the reason in `err`;
 * HDF5 features outside what the parser reads (dense link or attribute
 * storage, variable-length or compound data, chunk indexes other than the
 * version 1 B-tree and the single chunk, filters other than deflate / shuffle /
 * Fletcher-32) return GS_ERR_UNSUPPORTED. */
int gs_hdf_read_image(const char* path, int index, float** host_data, int* nx, int* ny, int* nz,
                      char* err, size_t err_len);
/* Any numeric dataset of an HDF5 file (user block allowed), converted to
 * double, row-major; dims[0..*rank-1] receive its extents (rank <= 8; a
 * scalar has rank 0 and one value).  Release with gs_host_free.  No reference
 * counterpart: an inspection helper over the same parser. */
int gs_hdf_read_dataset(const char* path, const char* dataset, double** host_data, int64_t* dims, int* rank,
                        char* err, size_t err_len);
/* Attribute `name` of the group or dataset `object`: numeric values (the
 * first max_values, converted to double; *n_values = their count) or, for a
 * fixed-length string, its text in `text`.  No reference counterpart. */
int gs_hdf_read_attribute(const char* path, const char* object, const char* name, double* values,
                          size_t max_values, size_t* n_values, char* text, size_t text_len, char* err,
                          size_t err_len);
void gs_host_free(void* p);

/* Correlation of one window with a set of templates, allocating nothing.
 * This entry point has no counterpart in the reference; it serves callers
 * that may not allocate device memory while they run (code being captured
 * into a CUDA graph, allocator-free real-time sections, hosts that hand the
 * library fixed buffers and forbid it to grow).  The caller passes device
 * buffers:
 *   d_window_spectrum  l x l complex (interleaved re, im float32): the window
 *                      spectrum as the search builds it (FFT / l^2, scaled);
 *   d_pair_spectra     ceil(n_templates/2) x l x l complex: for templates
 *                      2p and 2p+1, P_p = T_2p - i T_2p+1, T_j the spectrum
 *                      of normalised, rotated, masked template j (FFT / l^2);
 *   d_units            n_templates results (score, pos, peak, sigma) for
 *                      this window, as gs_get_units reports them.
 * The intermediate maps, accumulators and twiddles live in one static device
 * array of GS_NOALLOC_SCRATCH_BYTES that every GPU loading this library holds
 * until process exit; l is limited to GS_NOALLOC_MAX_WINDOW (odd l returns
 * GS_ERR_ARG; larger windows or l with too many prime factors return
 * GS_ERR_UNSUPPORTED).  Work is queued on `stream` (a cudaStream_t, NULL =
 * default stream) and the call returns without waiting.  The first call in
 * each CUDA context (per device, and again after that context is destroyed
 * and re-created, e.g. by cudaDeviceReset) looks up the array's device
 * address and must come before any stream capture.  All calls share the
 * array and it keeps the last call's contents: calls that overlap on the GPU
 * (other streams, other host threads) race. */
#define GS_NOALLOC_SCRATCH_BYTES (32u << 20)
#define GS_NOALLOC_MAX_WINDOW 2012
int gs_correlate_window_noalloc(const float* d_window_spectrum, const float* d_pair_spectra,
                                int n_templates, int l, float d_m, gs_unit* d_units, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* GISSPA_H */
