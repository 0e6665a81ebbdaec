/*
 * cbmv.h -- C ABI of libcbmv, the B200 (sm_100a) implementation of CBMV's
 * cost-volume path: matchers, feature extraction, random-forest classifier
 * and the MC-CNN cost optimisation ("post").
 *
 * The reference exposes this path as three boost.python modules imported by
 * its Python drivers (test.py:30-35, train.py:25-28):
 *   libmatchers    cpp/matchers/matchers.cpp:568-582
 *   libfeatextract cpp/featextract/featextract.cpp:519-540
 *   post           cpp/post/post.cu:905-933
 * plus scikit-learn's RandomForestClassifier.predict_proba (test.py:620).
 * Each entry point below names the reference function it replaces.  The
 * Python package cbmv_b200 binds these with ctypes under the reference's own
 * module and function names (cbmv_b200.libmatchers, .libfeatextract, .post).
 *
 * Conventions
 *  - Every pointer argument is DEVICE memory unless the comment says
 *    otherwise; the caller owns it.  Every call is asynchronous on `stream`
 *    (a cudaStream_t; NULL = the legacy default stream).
 *  - Every function returns 0 on success or a negative CBMV_E* code; the
 *    message of the last failure on the calling thread is cbmv_last_error().
 *    Invalid arguments are rejected on the host before anything is launched.
 *  - Volumes are dense and row-major.  CBMV_HWD = [H,W,D] (d fastest, the
 *    reference's census layout and the pipeline's internal layout);
 *    CBMV_DHW = [D,H,W] (the reference's nccNister/sadsob/zsad layout).
 *  - Invalid (border) cost entries hold the reference's sentinel RAND_MAX =
 *    2147483647 (2147483648.0f when stored as float32).
 *  - Sizes are int64; H*W*D may exceed 2^31.
 */
#ifndef CBMV_H_
#define CBMV_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* libcbmv.so is built with hidden visibility: the declarations of this
 * header are its only exported symbols. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

enum cbmv_status {
  CBMV_OK = 0,
  CBMV_EINVAL = -1,  /* bad argument (null pointer, size, window, dtype ...) */
  CBMV_ECUDA = -2,   /* a CUDA runtime call failed                          */
  CBMV_ENOMEM = -3,  /* device allocation failed                            */
  CBMV_ERANGE = -4,  /* size beyond a documented limit                      */
  CBMV_ESTATE = -5   /* object used in the wrong state                       */
};

enum cbmv_dtype { CBMV_F32 = 0, CBMV_F64 = 1 };
/* Hidden-layer activation of the learned classifier (cbmv_mlp_set_activation). */
enum cbmv_activation { CBMV_ACT_RELU = 0, CBMV_ACT_GELU = 1 };
/* 16-bit operand type of the network's fused inference (cbmv_mlp_set_precision). */
enum cbmv_precision { CBMV_PREC_F16 = 0, CBMV_PREC_BF16 = 1 };
enum cbmv_layout { CBMV_HWD = 0, CBMV_DHW = 1 };

/* Message of the last failed call on this thread ("" if none). */
const char* cbmv_last_error(void);
/* Library version, e.g. "cbmv-b200 0.1". */
const char* cbmv_version(void);
/* Waits for all work on `stream`. */
int cbmv_sync(void* stream);

/* ------------------------------------------------------------------ */
/* matchers -- libmatchers                                            */
/* ------------------------------------------------------------------ */

/* census (matchers.cpp:209-350): 121-bit (wsize^2) census descriptors,
 * Hamming cost for d <= column index of the window.  L, R: uint8 [H,W].
 * out: [H,W,D] or [D,H,W] of float32/float64.  wsize odd, wsize^2 <= 128. */
int cbmv_census(const uint8_t* L, const uint8_t* R, int64_t H, int64_t W, int D, int wsize,
                void* out, int dtype, int layout, void* stream);

/* census without any device allocation -- no counterpart in the reference.
 * Same arguments, results and errors as cbmv_census, for callers that may
 * not allocate device memory when they call the matcher (an arena or
 * caching allocator that owns the device heap, a CUDA graph being captured,
 * a plugin host that hands out only input and output buffers).  Its scratch
 * -- the two census descriptor images -- lives in one fixed device array of
 * cbmv_census_static_max_pixels() pixels per image (1,048,576; 32 MiB held
 * by every GPU that loads the library, until the process exits).  Larger
 * images are rejected with CBMV_ERANGE; use cbmv_census for them.
 *  - The first call on each device looks up the array's device address
 *    (cudaGetSymbolAddress); make that first call before any stream capture.
 *    The address is kept for the life of the process: a process that calls
 *    cudaDeviceReset on a device must not call this entry point afterwards.
 *  - All calls on a device share the one array: calls whose work overlaps on
 *    the GPU (different streams, or threads without ordering) race and
 *    corrupt each other's results; serialise them on one stream.
 *  - Each call writes every descriptor it reads, so no clearing is needed
 *    between calls. */
int cbmv_census_static(const uint8_t* L, const uint8_t* R, int64_t H, int64_t W, int D,
                       int wsize, void* out, int dtype, int layout, void* stream);
int64_t cbmv_census_static_max_pixels(void);

/* nccNister (matchers.cpp:24-205): normalised cross-correlation cost
 * -(w^2 S - A_L A_R) C_L C_R, 1 on flat windows.  wsize odd, <= 15. */
int cbmv_ncc(const uint8_t* L, const uint8_t* R, int64_t H, int64_t W, int D, int wsize,
             void* out, int dtype, int layout, void* stream);

/* sobel (matchers.cpp:515-555): horizontal Sobel response written at
 * (i+1, j+1) for i < H-3, j < W-3, zero elsewhere.  out [H,W] f32/f64. */
int cbmv_sobel(const uint8_t* img, int64_t H, int64_t W, void* out, int dtype, void* stream);

/* sadsob (matchers.cpp:353-436): box sum of |SL - SR(j-d)| over Sobel
 * responses SL, SR ([H,W], dtype sob_dtype, integer-valued).  wsize odd <= 15. */
int cbmv_sadsob(const void* SL, const void* SR, int sob_dtype, int64_t H, int64_t W, int D,
                int wsize, void* out, int dtype, int layout, void* stream);

/* zsad (matchers.cpp:440-512): zero-mean SAD.  wsize odd <= 15. */
int cbmv_zsad(const uint8_t* L, const uint8_t* R, int64_t H, int64_t W, int D, int wsize,
              void* out, int dtype, int layout, void* stream);

/* ------------------------------------------------------------------ */
/* feature extraction -- libfeatextract (float64 volumes, as the      */
/* reference's)                                                       */
/* ------------------------------------------------------------------ */

/* swap_axes (featextract.cpp:24-53): [D,H,W] -> [H,W,D]. */
int cbmv_swap_axes(const double* in, int64_t D, int64_t H, int64_t W, double* out, void* stream);
/* swap_axes_back (featextract.cpp:55-83): [H,W,D] -> [D,H,W]. */
int cbmv_swap_axes_back(const double* in, int64_t H, int64_t W, int64_t D, double* out,
                        void* stream);
/* get_cost (featextract.cpp:85-113): [H,W,D,K] -> [H,W,D], k = 0. */
int cbmv_get_cost(const double* in, int64_t H, int64_t W, int64_t D, int64_t K, double* out,
                  void* stream);
/* get_right_cost (featextract.cpp:115-152): R[i,j,d] = C[i,j+d,d], else C[0,0,0]. */
int cbmv_get_right_cost(const double* C, int64_t H, int64_t W, int64_t D, double* out,
                        void* stream);
/* get_left_cost (featextract.cpp:452-488): L[i,j,d] = R[i,j-d,d], else R[0,0,0]. */
int cbmv_get_left_cost(const double* Rv, int64_t H, int64_t W, int64_t D, double* out,
                       void* stream);
/* extract_ratio, test form (featextract.cpp:303-342): rows of [N,D]. */
int cbmv_extract_ratio(const double* vol, int64_t N, int64_t D, double e, double* out,
                       void* stream);
/* extract_likelihood, test form (featextract.cpp:402-450). */
int cbmv_extract_likelihood(const double* vol, int64_t N, int64_t D, double sigma, double* out,
                            void* stream);
/* extract_ratio, training form (featextract.cpp:254-300): samples int32 [N,3]; out [3N]. */
int cbmv_extract_ratio_samples(const double* vol, int64_t N, int64_t D, const int32_t* samples,
                               double e, double* out, void* stream);
/* extract_likelihood, training form (featextract.cpp:345-399). */
int cbmv_extract_likelihood_samples(const double* vol, int64_t N, int64_t D,
                                    const int32_t* samples, double sigma, double* out,
                                    void* stream);
/* get_samples (featextract.cpp:217-252). */
int cbmv_get_samples(const double* vol, int64_t N, int64_t D, const int32_t* samples,
                     double* out, void* stream);
/* generate_labels (featextract.cpp:490-516): [1,0,0] per sample; out int32 [3N]. */
int cbmv_generate_labels(int64_t N, int32_t* out, void* stream);
/* generate_d_indices (featextract.cpp:154-215): one positive (gt) and two
 * negatives per sample drawn |d - gt| > thr from a counter-based generator
 * keyed by `seed` (the reference's rand() under OpenMP is not reproducible).
 * gt int32 [N] with 0 <= gt <= maxd; out int32 [N,3].  CBMV_EINVAL when a
 * sample's range is empty (where the reference divides by zero). */
int cbmv_generate_d_indices(const int32_t* gt, int64_t N, int maxd, int thr, uint64_t seed,
                            int32_t* out, void* stream);

/* Fused features (test.py:521-595, Testing.__extract_features_lr): the 20
 * CBMV features per (pixel, d) from the four [H,W,D] float64 cost volumes
 * (census, ncc, sadsob, zsad, in that order), column order as the reference:
 * 0-3 costs, 4-7 ratio, 8-11 likelihood, 12-15 right-reference ratio warped
 * to the left view, 16-19 the same for likelihood.  Computed in float64 as
 * the reference and stored as float32 (what the random forest reads).
 * out float32 [H*W*D, 20]. */
int cbmv_features(const double* census, const double* ncc, const double* sob, const double* sad,
                  int64_t H, int64_t W, int D, float* out, void* stream);

/* ------------------------------------------------------------------ */
/* random forest -- sklearn RandomForestClassifier.predict_proba      */
/* ------------------------------------------------------------------ */

typedef struct cbmv_forest cbmv_forest;

/* Uploads a packed forest (HOST pointers; layout in cbmv_b200/forest.py and
 * csrc/rf.cuh): blocks uint32 [n_blocks,8] -- each 32-byte block holds two
 * tree levels -- leaf_value float64 [n_leaves,2] (class-0 and class-1
 * fractions), tree_offsets int32 [n_trees+1] (first block of each tree).
 * The structure is validated on the host (CBMV_EINVAL on any index out of
 * range).  Replaces unpickling the sklearn model (test.py:603-604). */
int cbmv_forest_create(const uint32_t* blocks, int64_t n_blocks, const double* leaf_value,
                       int64_t n_leaves, const int32_t* tree_offsets, int n_trees,
                       int n_features, cbmv_forest** out);
/* Sizes of an uploaded forest. */
int cbmv_forest_info(const cbmv_forest* f, int* n_trees, int64_t* n_blocks, int64_t* n_leaves);
int cbmv_forest_destroy(cbmv_forest* f);

/* predict_proba (sklearn/ensemble/_forest.py ForestClassifier.predict_proba,
 * called at test.py:620): X float32 [N,F]; proba float64 [N,2] (may be
 * NULL): column k = sum over trees, in tree order, of the leaf's class-k
 * fraction, / n_trees.  leaves int32 [N,n_trees] (may be NULL): the leaf
 * reached in each tree, as an index into leaf_value (FlatForest.pack
 * returns the map back to sklearn's node ids). */
int cbmv_forest_predict(const cbmv_forest* f, const float* X, int64_t N, double* proba,
                        int32_t* leaves, void* stream);

/* ------------------------------------------------------------------ */
/* learned classifier (MLP surrogate of the random forest)             */
/* ------------------------------------------------------------------ */

/* C[M,N] (float32) = A[M,K] * B[N,K]^T on the tcgen05 tensor cores, A and B
 * bfloat16 row-major (K contiguous), all 16-byte aligned; M % 128 == 0,
 * N % 32 == 0, K % 64 == 0.  *status (device int) is set to 1 if a
 * tensor-core completion wait timed out (the result is then invalid). */
int cbmv_gemm_bf16(const uint16_t* A, const uint16_t* B, float* C, int64_t M, int64_t N, int64_t K,
                   int* status, void* stream);

/* The classifier network: 20 -> 128 -> 128 -> 64 -> 1, GELU or ReLU hidden
 * layers (cbmv_mlp_set_activation; ReLU when created), sigmoid output =
 * P(correct match); its matching cost is 1 - P.  Its
 * parameter vector (float32, cbmv_mlp_num_params() values) is, in order:
 * cap[20], mu[20], inv_sd[20] (input transform x' = (min(x,cap)-mu)*inv_sd),
 * W1[128x20], b1[128], W2[128x128], b2[128], W3[64x128], b3[64], w4[64],
 * b4.  Training runs on the tcgen05 GEMM above with bfloat16 activations and
 * float32 accumulation, float32 master weights and Adam. */
typedef struct cbmv_mlp cbmv_mlp;
int cbmv_mlp_num_params(void);
/* batch: samples per training step, a multiple of 128. */
int cbmv_mlp_create(int batch, cbmv_mlp** out);
int cbmv_mlp_destroy(cbmv_mlp* m);
/* Parameters from / to HOST memory; setting them resets the optimiser. */
int cbmv_mlp_set_params(cbmv_mlp* m, const float* host_params);
int cbmv_mlp_get_params(const cbmv_mlp* m, float* host_params);
/* One Adam step (betas 0.9/0.999, decoupled weight decay) on X float32
 * [batch,20] raw features and y float32 [batch] labels (device memory);
 * loss (device float, may be NULL) receives the mean binary cross-entropy. */
int cbmv_mlp_train_step(cbmv_mlp* m, const float* X, const float* y, float lr, float weight_decay,
                        float* loss, void* stream);
/* Loss gradients in parameter order without the input transform
 * (num_params - 60 floats, device memory), no update. */
int cbmv_mlp_gradients(cbmv_mlp* m, const float* X, const float* y, float* grads, float* loss,
                       void* stream);
/* 0 while every tensor-core completion wait has succeeded. */
int cbmv_mlp_status(const cbmv_mlp* m, int* status);
/* Hidden-layer activation, CBMV_ACT_RELU or CBMV_ACT_GELU, used by training
 * and by the fused inference of cbmv_run_mlp alike.  The GELU is x * Phi(x)
 * evaluated in IEEE half-precision operations as x * clamp(0.5 + x p(x^2),
 * 0, 1) with a fixed quadratic p (within 8.32e-3 of the exact erf form on
 * every finite f16 x; the polynomial itself is within 7.7e-3); it runs on
 * the packed half-precision FMA pipe, not the special-function unit.  The
 * fused inference runs the network on f16 operands (inputs, weights,
 * activations; float32 accumulation, biases as f16 high + low parts).  No
 * counterpart in the reference (its classifier is the random forest). */
int cbmv_mlp_set_activation(cbmv_mlp* m, int act);
int cbmv_mlp_get_activation(const cbmv_mlp* m, int* act);
/* Operand type of the fused inference (cbmv_run_mlp): CBMV_PREC_F16 (when
 * created) or CBMV_PREC_BF16, both with float32 accumulation, biases as
 * 16-bit high + low parts.  The bf16 form evaluates the GELU's polynomial
 * in bf16 operations with its own coefficients (within 1.21e-2 of
 * x * Phi(x) on every bf16 x, seven instructions per pair of columns against
 * six in f16, whose saturating FMA folds the clamp).  Training always runs
 * on bf16 GEMM operands. */
int cbmv_mlp_set_precision(cbmv_mlp* m, int prec);
int cbmv_mlp_get_precision(const cbmv_mlp* m, int* prec);

/* ------------------------------------------------------------------ */
/* cost optimisation -- post (post.cu), float32 on the device          */
/* ------------------------------------------------------------------ */

/* cross (post.cu:336-396): out float32 [4,H,W] arm end coordinates. */
int cbmv_cross(const float* img, int64_t H, int64_t W, int L1, float tau1, float* out,
               void* stream);
/* sgm_w (post.cu:263-333): out += sum over the 4 scan directions of the
 * path costs of `in` ([H,W,D] float32).  `out` is NOT cleared (the reference
 * zeroes it first, test.py:379).  D <= 1024. */
int cbmv_sgm(const float* imL, const float* imR, const float* in, int64_t H, int64_t W, int D,
             float pi1, float pi2, float tau_so, float alpha1, float q1, float q2, int direction,
             float* out, void* stream);
/* cbca (post.cu:399-450) on a volume of layout `layout`; in != out. */
int cbmv_cbca(const float* crossL, const float* crossR, const float* in, int64_t H, int64_t W,
              int D, int layout, int direction, float* out, void* stream);
/* cbca of the same arms and volume in separable form (row sums, then column
 * sums of each support; the fused pipeline's default): [H,W,D] layout only,
 * arms from cbmv_cross with the same L1 (2..9); in != out.  Equal to
 * cbmv_cbca up to float rounding.  With L1 <= 6 the supports are first
 * stored as one 32-bit word per (p,d) in a stream-ordered scratch buffer
 * (cudaMallocAsync / cudaFreeAsync on `stream`, 4 B per (p,d)); the result
 * is bit-identical either way. */
int cbmv_cbca_separable(const float* crossL, const float* crossR, const float* in, int64_t H,
                        int64_t W, int D, int L1, int direction, float* out, void* stream);
/* np.argmin over d (test.py:408-409), first minimum; disp float32 [H,W]. */
int cbmv_wta(const float* cost, int64_t H, int64_t W, int D, int layout, float* disp,
             void* stream);
/* subpixel_enchancement (post.cu:453-483). */
int cbmv_subpixel(const float* disp, const float* cost, int64_t H, int64_t W, int D, int layout,
                  float* out, void* stream);
/* median2d (post.cu:486-518), k odd <= 11. */
int cbmv_median2d(const float* in, int64_t H, int64_t W, int k, float* out, void* stream);
/* mean2d (post.cu:520-566): kernel float32 [ks,ks] in DEVICE memory, ks odd <= 31. */
int cbmv_mean2d(const float* in, int64_t H, int64_t W, const float* kernel, int ks, float alpha2,
                float* out, void* stream);
/* outlier_detection (post.cu:717-754). */
int cbmv_outlier_detection(const float* d0, const float* d1, int64_t H, int64_t W, int disp_max,
                           float* out, void* stream);
/* interpolate_mismatch (post.cu:757-827). */
int cbmv_interpolate_mismatch(const float* d0, const float* outlier, int64_t H, int64_t W,
                              float* out, void* stream);
/* interpolate_occlusion (post.cu:829-869). */
int cbmv_interpolate_occlusion(const float* d0, const float* outlier, int64_t H, int64_t W,
                               float* out, void* stream);
/* Volume helpers replacing post.swap_axis / swap_axis_back / CUDA_divide_double
 * (post.cu:569-684) on float32 volumes. */
int cbmv_transpose_f32(const float* in, int64_t H, int64_t W, int64_t D, int to_layout,
                       float* out, void* stream);
int cbmv_scale_f32(float* a, int64_t n, float mul, void* stream);
/* float64 <-> float32 conversion of n elements. */
int cbmv_f64_to_f32(const double* in, int64_t n, float* out, void* stream);
int cbmv_f32_to_f64(const float* in, int64_t n, double* out, void* stream);

/* ------------------------------------------------------------------ */
/* end-to-end pipeline                                                 */
/* ------------------------------------------------------------------ */

/* Parameters of Testing.__init__ (test.py:44-73) and the feature constants
 * (test.py:71-73, 548-551); cbmv_params_default fills the reference's
 * defaults. */
typedef struct cbmv_params {
  int censw, nccw, sadw, sobw;
  float pi1, pi2, sgm_q1, sgm_q2, alpha1, tau_so;
  int sgm_i;
  int L1;
  float tau1;
  int cbca_i1, cbca_i2, median_i, median_w;
  float blur_sigma, blur_t;
  int direction;
  /* CBCA summation: 0 (default) row sums then column sums of each support
   * (separable form, rounding differs from the reference's); 1 one running
   * float sum per support in the reference's order (post.cu:415-429). */
  int exact_cbca;
  /* Most CTAs (one per SM) the learned classifier's kernel may occupy;
   * 0 = every SM.  Lower values leave SMs to pairs running concurrently
   * (cbmv_batch). */
  int mlp_ctas;
  /* Launch shapes that do not change the results (picked by the batch
   * autotuner): rows per CBCA tile, 16 or 32 (0 = 32); SGM steps loaded
   * ahead, 1, 2 or 4 (0 = the default for the disparity count). */
  int cbca_rows, sgm_prefetch;
  /* Post-processing chain, Testing.eval_prob's `interpolate` (main.py:70,
   * test.py:143-149): 0 (default) the _mem post (test.py:341-449); 1 the
   * _interp post (test.py:153-338): the right view's cost
   * (get_right_cost) through the same chain with the arms swapped and the
   * direction negated, then the left-right check (outlier_detection) and
   * its fills (interpolate_mismatch, interpolate_occlusion) on the left
   * view's integer winner-take-all disparity, as the reference's chain
   * does (its subpixel result is overwritten, test.py:293-300); median and
   * blur follow.  Needs one more float32 [H,W,D] volume of workspace.
   * cbmv_batch_run_mlp accepts 0 only. */
  int interpolate;
} cbmv_params;
void cbmv_params_default(cbmv_params* p);

typedef struct cbmv_ctx cbmv_ctx;

/* A context owns the device workspaces of one pair shape and one stream;
 * it grows them on demand.  Not thread-safe: one context per host thread.
 * Inside cbmv_run_rf / cbmv_run_mlp / cbmv_run_post some independent work
 * (the post's image terms beside the matchers, the CBCA supports beside the
 * SGM) runs on a second stream the context creates; events order it with
 * `stream` both ways, so every call's work is complete once `stream` has
 * passed the call (also under stream capture). */
int cbmv_ctx_create(void* stream, cbmv_ctx** out);
int cbmv_ctx_destroy(cbmv_ctx* c);

/* The reference's test path for one rectified pair (main.py:53-70 with
 * interpolate=False): matchers -> features -> random forest -> P(class 0)
 * -> post (_mem chain, test.py:341-449) -> disparity.  L, R uint8 [H,W],
 * disp float32 [H,W], all device memory.  prob0 (optional, may be NULL)
 * receives the float32 [H,W,D] matching-cost volume P(class 0). */
int cbmv_run_rf(cbmv_ctx* c, const cbmv_forest* f, const cbmv_params* p, const uint8_t* L,
                const uint8_t* R, int64_t H, int64_t W, int D, float* disp, float* prob0);

/* The same path with the learned classifier in place of the forest: the
 * network's matching cost 1 - P(correct) feeds the post-processing.  The
 * features and the network run fused on the tensor cores (no feature matrix
 * in HBM).  Tensor-core wait timeouts are reported by cbmv_mlp_status. */
int cbmv_run_mlp(cbmv_ctx* c, const cbmv_mlp* m, const cbmv_params* p, const uint8_t* L,
                 const uint8_t* R, int64_t H, int64_t W, int D, float* disp, float* prob0);

/* cbmv_run_rf / cbmv_run_mlp with HOST buffers, the form a driver holding
 * its images in host memory binds (the reference's drivers pass numpy
 * arrays to its modules and read the disparity on the host,
 * test.py:143-149, 408-409): L, R uint8 [H,W] and disp float32 [H,W] in
 * host memory, pinned or pageable.  The images are copied into device
 * buffers the context owns (grown on demand, freed with it), the path
 * runs on the context's stream, the disparity is copied back, and the
 * call returns once it is in `disp` (the stream is synchronised).  Errors
 * as the device-pointer forms; W <= 2^24. */
int cbmv_run_rf_host(cbmv_ctx* c, const cbmv_forest* f, const cbmv_params* p, const uint8_t* L,
                     const uint8_t* R, int64_t H, int64_t W, int D, float* disp);
int cbmv_run_mlp_host(cbmv_ctx* c, const cbmv_mlp* m, const cbmv_params* p, const uint8_t* L,
                      const uint8_t* R, int64_t H, int64_t W, int D, float* disp);

/* The post-processing alone (Testing.eval_prob with the _mem chain,
 * test.py:143-149, 341-449) on a given matching cost: cost float32 [H,W,D]
 * (low = good, e.g. a saved P(class 0) volume, main.py:56-67), the images L,
 * R uint8 [H,W] for the cross arms and SGM, disp float32 [H,W]; device
 * memory.  `cost` is not modified. */
int cbmv_run_post(cbmv_ctx* c, const cbmv_params* p, const uint8_t* L, const uint8_t* R, int64_t H,
                  int64_t W, int D, const float* cost, float* disp);

/* The four float32 matcher volumes of the learned path (census, NCC,
 * SAD-on-Sobel, ZSAD; the reference's test.py:122-138 costs, [H,W,D]
 * layout) into out float32 [4,H,W,D], device memory.  Census, NCC and
 * SAD-on-Sobel equal the float32 rounding of the reference's values; ZSAD is
 * the exact window quotient, within one float32 unit of it. */
int cbmv_ctx_volumes_f32(cbmv_ctx* c, const cbmv_params* p, const uint8_t* L, const uint8_t* R,
                         int64_t H, int64_t W, int D, float* out);

/* Training-sample emission (the GPU counterpart of train.py:100-273): the
 * 20 float32 features of the samples idx[i] = (y*W + x)*D + d of the pair
 * (L, R); idx int64 [n], out float32 [n,20], device memory. */
int cbmv_ctx_features_at(cbmv_ctx* c, const cbmv_params* p, const uint8_t* L, const uint8_t* R,
                         int64_t H, int64_t W, int D, const int64_t* idx, int64_t n, float* out);

/* The learned path's own 20 features of the samples idx[i] = (y*W + x)*D + d
 * (the float32 arithmetic the fused network kernel of cbmv_run_mlp forms
 * them with, from its float32 volumes and row statistics; the reference's
 * are float64, test.py:521-595): idx int64 [n], out float32 [n,20], device
 * memory. */
int cbmv_ctx_features_f32_at(cbmv_ctx* c, const cbmv_params* p, const uint8_t* L, const uint8_t* R,
                             int64_t H, int64_t W, int D, const int64_t* idx, int64_t n, float* out);

/* ------------------------------------------------------------------ */
/* batches of pairs of uneven size                                     */
/* ------------------------------------------------------------------ */

/* A batch of n pairs (H[i] x W[i], D[i] disparities) run by the learned
 * path as ONE CUDA graph launch: the pairs are spread over `streams`
 * concurrent contexts (longest first onto the least-loaded context), each
 * with a workspace sized for its largest pair; the graph holds every pair's
 * kernels, a fork/join over the contexts and per-pair timing events.  No
 * counterpart in the reference, which runs one pair per process
 * (main.py:53-70).  Creation allocates the workspaces. */
typedef struct cbmv_batch cbmv_batch;
int cbmv_batch_create(int n, const int64_t* H, const int64_t* W, const int* D, int streams,
                      cbmv_batch** out);
int cbmv_batch_destroy(cbmv_batch* b);
/* Runs the batch on `stream`: L[i], R[i] uint8 [H[i],W[i]], disp[i] float32
 * [H[i],W[i]], device memory.  The first call (and any call whose pointers,
 * network or parameters differ from the previous one) captures the graph;
 * the others replay it.  Asynchronous. */
int cbmv_batch_run_mlp(cbmv_batch* b, const cbmv_mlp* m, const cbmv_params* p, const uint8_t* const* L,
                       const uint8_t* const* R, float* const* disp, void* stream);
/* After the last run has completed: pair_ms[i] = time from pair i's first
 * kernel to its last, done_ms[i] = time from the graph's start to pair i's
 * end, *total_ms = the graph's span (all ms). */
int cbmv_batch_timings(cbmv_batch* b, float* pair_ms, float* done_ms, float* total_ms);

/* Stage timings of the last cbmv_run_* call in milliseconds (CUDA events):
 * [0] matchers, [1] feature statistics, [2] features+classifier, [3] post,
 * [4] total.  Valid after the stream has been synchronised. */
int cbmv_ctx_timings(cbmv_ctx* c, float* ms5);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif
#endif /* CBMV_H_ */
