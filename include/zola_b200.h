/*
 * zola_b200.h — C-ABI of the B200-native ZOLA-3D localization library.
 *
 * This is the whole boundary: plain pointers and sizes, no C++ or torch types.
 * It replaces the JCuda object API that ZOLA-3D's Java classes drive (paths are
 * relative to the reference's src/main/java/org/pasteur/imagej/):
 *
 *   MyCudaStream.init / destroy                 cuda/MyCudaStream.java:36-132
 *   DataPhase_ (+ PSFmany_float_ construction)  process/gpu/DataPhase_.java,
 *                                               process/gpu/PSFmany_float_.java:186-500
 *   PSFmany_float_.computePSF                   process/gpu/PSFmany_float_.java:1626-1720
 *   Modelmany_double_.getLikelihood / Fisher    process/gpu/Modelmany_double_.java:545-791,865-940
 *   Localization_.localize (per-ROI MLE)        process/gpu/Localization_.java:633-798
 *
 * Conventions (all functions):
 *   - return 0 on success, a negative ZOLA_E* code on failure; zola_last_error()
 *     gives a message.  The reference logged and continued (IJ.log); here every
 *     failure is reported to the caller.
 *   - x, y, z, pixel size and wavelength are in micrometres; Zernike
 *     coefficients are in radians, un-normalised, in the reference's index order
 *     (n = 0,1,2,..., m = -n,-n+2,...,n; utils/Zernike.java:26-60).
 *   - images and ROIs are stored [x][y] (first index x), as the reference's
 *     double[][] arrays (process/cpu/LocalizationPipeline.java:588-606).
 *   - "host" entry points take host buffers and copy in and out inside the call;
 *     "_dev" entry points take device pointers and a cudaStream_t (as void*).
 *   - a context is not thread-safe; use one per host thread (the reference's
 *     "part"/stream), exactly as the reference used one DataPhase_ per stream.
 */
#ifndef ZOLA_B200_H
#define ZOLA_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define ZOLA_API __attribute__((visibility("default")))
#else
#define ZOLA_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define ZOLA_OK 0
#define ZOLA_E_ARG -1       /* invalid argument (size, null pointer, range) */
#define ZOLA_E_CUDA -2      /* CUDA runtime error */
#define ZOLA_E_NODEV -3     /* no usable sm_100 device */
#define ZOLA_E_UNSUPPORTED -4
#define ZOLA_E_TIMEOUT -5   /* a bounded device wait ran out (kernel status word) */

typedef struct zola_ctx zola_ctx;
typedef struct zola_psf zola_psf;

/* Optical parameters of one calibration (the calibration JSON keys of
 * process/cpu/DataPhase.java:587-679 plus the localization command's n_wat). */
typedef struct {
    int size_fft;        /* "sizeFFT": pupil grid; made even and rounded up to a
                            power of two as the CPU path does (PhaseParameters.java:296) */
    double xystep;       /* "sizePix", um */
    double na;           /* "NA" */
    double wavelength;   /* "wavelength", um */
    double n_oil;        /* "index" (immersion) */
    double n_wat;        /* sample index (DataPhase.setNwat) */
    double sigma;        /* "sigmaGaussianKernel", px */
    int with_apo;        /* "withApoFactor" */
    double zfocus;       /* Zfocus: the zoil the localization model uses, um */
    int kz_reset;        /* 1: evanescent kz = 2 pi sqrt|.| as PSFPhase.resetKz
                            (detection library); 0: kz = 0 (fit model, PSFPhaseMany) */
} zola_optics;

/* Levenberg-Marquardt fit controls. */
typedef struct {
    double zmin, zmax;   /* z box, um (reference: minZ-0.3, maxZ+0.3) */
    double xymax;        /* |x|,|y| box, um */
    int max_iter;        /* model evaluations per ROI (config: 30) */
    double tol_xyz;      /* convergence: accepted step below this, um */
    double step_xy;      /* per-iteration step caps, um */
    double step_z;
    int precision;       /* ZOLA_PREC_* */
} zola_fit_params;

#define ZOLA_PREC_FP64 0     /* plain FP64 GPU form (CUDA cores, one CTA per ROI) */
#define ZOLA_PREC_SPLIT 1    /* split-precision tcgen05 partial DFT, FP32 sums, FP64 solve */

/* Per-ROI status codes written by the fits. */
#define ZOLA_FIT_CONVERGED 1
#define ZOLA_FIT_MAXITER 2
#define ZOLA_FIT_STALLED 3
#define ZOLA_FIT_NAN -1

/* --- context (replaces MyCudaStream.init / destroy, cuda/MyCudaStream.java:36-132).
 * Free every PSF of a context (zola_psf_free) before destroying the context. */
ZOLA_API int zola_ctx_create(int device, zola_ctx** out);
ZOLA_API int zola_ctx_destroy(zola_ctx* ctx);
ZOLA_API const char* zola_last_error(const zola_ctx* ctx);
/* Stream the context launches on (cudaStream_t as void*).  The *_dev entry
 * points take a stream argument; NULL means this stream.  It is a blocking
 * stream, so CUDA orders it with the legacy default stream (stream 0, torch's
 * default stream): device inputs written there before the call are complete
 * when the call reads them, and work queued there after the call waits for it.
 * With any other stream of the caller's, pass that stream. */
ZOLA_API void* zola_ctx_stream(zola_ctx* ctx);

/* --- PSF (replaces DataPhase_ + PSFmany_float_ construction; the Java side
 * parses the unchanged calibration JSON and passes its fields here).
 * zernike: nz coefficients in radians (DataPhase.java:641-660). */
ZOLA_API int zola_psf_load(zola_ctx* ctx, const zola_optics* optics, const double* zernike, int nz,
                  zola_psf** out);
ZOLA_API int zola_psf_free(zola_psf* psf);
/* Grid facts: rounded pupil grid N and disk pixel count K. */
ZOLA_API int zola_psf_info(const zola_psf* psf, int* N, int* K);

/* --- PSF model (replaces PSFmany_float_.computePSF, PSFmany_float_.java:1626-1720,
 * and PSFPhase.computePSF, process/cpu/PSFPhase.java:557-629).
 * xyz: n triples (x, y, zwat) um, zoil = optics.zfocus.  out_psf: n*R*R FP64,
 * normalised to sum 1.  out_dpsf (nullable): n*3*R*R, d psi / d{x,y,z}.
 * FP64 on the device. */
ZOLA_API int zola_psf_model(zola_psf* psf, int R, const double* xyz, int n, double* out_psf, double* out_dpsf);
ZOLA_API int zola_psf_model_dev(zola_psf* psf, int R, const double* d_xyz, int n, double* d_out_psf,
                       double* d_out_dpsf, void* stream);
/* Same with an explicit arithmetic: ZOLA_PREC_FP64 (CUDA cores, FP64) or
 * ZOLA_PREC_SPLIT (the tcgen05 split-precision stages the split fit uses). */
ZOLA_API int zola_psf_model_prec(zola_psf* psf, int R, const double* xyz, int n, double* out_psf, double* out_dpsf,
                                 int precision);
ZOLA_API int zola_psf_model_prec_dev(zola_psf* psf, int R, const double* d_xyz, int n, double* d_out_psf,
                                     double* d_out_dpsf, int precision, void* stream);

/* --- batched Poisson MLE fit (replaces Localization_.localize with its
 * Modelmany_double_ likelihood batches, process/gpu/Localization_.java:633-798).
 * rois: n*R*R photon counts [x][y]; init5/out5: n*(x, y, z, A, B);
 * crlb5 (nullable): sqrt(diag(F^-1)) at the optimum, n*5; nll: n (deviance
 * form sum mu - d - d ln(mu/d)); status/iters: n (model evaluations). */
ZOLA_API int zola_fit_batch(zola_ctx* ctx, zola_psf* psf, int R, const float* rois, const double* init5, int n,
                   const zola_fit_params* prm, double* out5, double* crlb5, double* nll, int* status,
                   int* iters);
ZOLA_API int zola_fit_batch_dev(zola_ctx* ctx, zola_psf* psf, int R, const float* d_rois, const double* d_init5,
                       int n, const zola_fit_params* prm, double* d_out5, double* d_crlb5, double* d_nll,
                       int* d_status, int* d_iters, void* stream);
/* Streaming form of zola_fit_batch_dev for a producer that writes ROIs into
 * d_rois while the fit runs (replaces the detection -> localization hand-off of
 * LocalizationPipeline_'s producer and consumer threads,
 * process/gpu/LocalizationPipeline_.java:164-441): ROIs [0, *d_avail) are on
 * the device, and the producer raises the device int *d_avail (never lowers
 * it, up to n) as it writes more, with its writes made visible before the count
 * (e.g. a stream-ordered copy, or a release store).  Split precision; runs the
 * dataflow kernel.  If the count stops short of n, the call ends with
 * ZOLA_E_TIMEOUT once no ROI has arrived for the wait limit
 * (zola_ctx_set_wait_limit); every ROI below the count is fitted by then. */
ZOLA_API int zola_fit_batch_stream_dev(zola_ctx* ctx, zola_psf* psf, int R, const float* d_rois,
                                       const double* d_init5, const int* d_avail, int n, const zola_fit_params* prm,
                                       double* d_out5, double* d_crlb5, double* d_nll, int* d_status, int* d_iters,
                                       void* stream);

/* Mixed batch: several ROI classes (PSF and ROI side, e.g. 16 x 16 astigmatic,
 * 24 x 24 saddle and 48 x 48 tetrapod ROIs) fitted in one call (replaces the
 * reference's per-size Modelmany_double_ batches run side by side by its
 * worker threads, process/gpu/Modelmany_double_.java:865-940).  Each class has
 * its own slot pool and stream, and the classes' LM rounds are interleaved so
 * that one class's draining tail overlaps the others' work; each ROI's fit is
 * the same bit for bit as in a call of its class alone.  Device buffers as in
 * zola_fit_batch_dev; every class must use split precision. */
#define ZOLA_MAX_CLASSES 8
typedef struct {
    zola_psf* psf;
    int R, n;
    const float* d_rois;
    const double* d_init5;
    zola_fit_params prm;
    double *d_out5, *d_crlb5, *d_nll;  /* d_crlb5, d_nll nullable */
    int *d_status, *d_iters;           /* nullable */
} zola_fit_class;
ZOLA_API int zola_fit_batch_mixed_dev(zola_ctx* ctx, const zola_fit_class* classes, int nclass, void* stream);
/* Host-buffer form of the mixed batch: the d_* fields of each class point to
 * HOST memory here (pinned memory lets the copies overlap the fits).  Every
 * class is checked first; the ROIs then go up on the context's copy stream in
 * chunks of about 32 MB, interleaved across the classes, and each class starts
 * fitting on its first chunk and takes the others as they land.  The results
 * come back before the call returns and equal those of
 * zola_fit_batch_mixed_dev bit for bit. */
ZOLA_API int zola_fit_batch_mixed(zola_ctx* ctx, const zola_fit_class* classes, int nclass);

/* sCMOS form (process/cpu/Localization.java:1132, utils/SCMOScamera.java):
 * scmos holds, per ROI pixel, var/gain^2 of the camera pixel; it is added to
 * the model mean (mu = A psi + B + scmos), and rois are then
 * (ADU - offset)/gain + var/gain^2 as the reference converts them. */
ZOLA_API int zola_fit_batch_scmos(zola_ctx* ctx, zola_psf* psf, int R, const float* rois, const float* scmos,
                                  const double* init5, int n, const zola_fit_params* prm, double* out5, double* crlb5,
                                  double* nll, int* status, int* iters);
ZOLA_API int zola_fit_batch_scmos_dev(zola_ctx* ctx, zola_psf* psf, int R, const float* d_rois, const float* d_scmos,
                                      const double* d_init5, int n, const zola_fit_params* prm, double* d_out5,
                                      double* d_crlb5, double* d_nll, int* d_status, int* d_iters, void* stream);

/* --- detection (replaces Predetection / Predetection_cross_: library build,
 * setImage and convolveNormalizedInFourierDomain; process/cpu/Predetection.java:63-593,
 * process/gpu/Predetection_cross_.java:104-785).  psf must be built with
 * kz_reset = 1 (the reference builds its library from DataPhase.psf after
 * setNwat).  Library: ceil((maxZ-minZ)/step) slices at z = minZ + k*step
 * (accumulated), R x R each; thr is the NCC threshold (reference: 0.1). */
typedef struct zola_detector zola_detector;
ZOLA_API int zola_detector_create(zola_psf* psf, int SX, int SY, int R, double minZ, double maxZ, double step,
                                  double thr, zola_detector** out);
ZOLA_API int zola_detector_free(zola_detector* det);
/* Number of slices; optionally their z (um) and the normalised library PSFs
 * (nslices x R x R, sum 1), as Predetection.getRange / getPSFNonNormalized. */
ZOLA_API int zola_detector_info(const zola_detector* det, int* nslices, double* range, double* psfs);
/* frames: nframes x SX x SY photons (double, first index x).  out: nframes x
 * cap rows of 7 doubles (score, slice r, i, j, dz, dx, dy): the first
 * min(counts[f], cap) entries of frame f's whole candidate list, sorted by
 * descending score with ties in the reference's insertion order (slice r,
 * then j, then i; Predetection.getVectMaxPosition).  counts[f] = length of the
 * whole list (at 0.1, the reference's threshold, a 256 x 256 frame against a
 * 41-slice library gives several thousand). */
#define ZOLA_DETECT_MAX_CAP (1 << 20)
ZOLA_API int zola_detect(zola_detector* det, const double* frames, int nframes, int cap, double* out, int* counts);
/* Camera-count form: frames are nframes x SX x SY uint16 counts as the camera
 * writes them (2 bytes a pixel over the host link), turned into photons on
 * the device as LocalizationPipeline.java:601-605 does: count * (adu / gain) +
 * (-offset * adu / gain), negative values set to 0 (adu, gain, offset: the
 * arguments of the LocalizationPipeline constructor, :100-107). */
ZOLA_API int zola_detect_u16(zola_detector* det, const uint16_t* frames, int nframes, int cap, double adu,
                             double gain, double offset, double* out, int* counts);
/* Device form, asynchronous on stream: cap is also the number of candidates
 * stored per frame, so a frame with counts[f] > cap gets the sorted first cap
 * of its list in insertion order -- the same rows on every run, but not the
 * first cap of the sorted whole.  Call again with cap >= counts[f] for those. */
ZOLA_API int zola_detect_dev(zola_detector* det, const double* d_frames, int nframes, int cap, double* d_out,
                             int* d_counts, void* stream);

/* --- frame localization pipeline (replaces LocalizationPipeline_ / the
 * detect -> localize -> filter loop; process/cpu/LocalizationPipeline.java:145-1250).
 * One row per accepted localization, in the ThunderStorm CSV units. */
typedef struct {
    int id, frame;
    double x_nm, y_nm, z_nm;        /* 1000 * (pixel * dx - x) as the reference writes them */
    double intensity, background;   /* photons, photons / px */
    double chi2;                    /* scoreCompute: mean (patch - model)^2 / model */
    double crlb_x_nm, crlb_y_nm, crlb_z_nm;
    int candidate;                  /* index of the row's candidate in its frame's sorted candidate list */
    int fit_status;                 /* the fit's status: 1 converged, 2 evaluation cap, 3 stalled */
} zola_localization;

typedef struct {
    int patch;                /* ROI side R; must equal the detector's R */
    double minZ, maxZ;        /* accepted z range (ZfocusCenter -/+ axialRange/2); the fit box is 0.3 um wider */
    double photon_threshold;  /* photonThreshold */
    double max_snr;           /* maxSNR (reference: 1) */
    int max_iter;             /* LM evaluations per ROI */
    double tol_xyz;           /* LM stopping distance, um */
    int precision;            /* ZOLA_PREC_FP64 or ZOLA_PREC_SPLIT for the fits */
    int cand_cap;             /* candidates stored per frame at the start (0: 8192); it grows to the
                                 longest list so that every frame walks its whole list */
    int frames_per_batch;     /* frames per device batch (0: 1024) */
    int wave_fits;            /* candidates fitted ahead per frame and wave (0: 8); any value gives the
                                 same rows as the reference's one-at-a-time walk */
} zola_loc_params;

/* frames: nframes x SX x SY photons (double, first index x, already converted
 * with the camera ADU / gain / offset and clamped at 0 as the reference does).
 * det: a detector on a kz_reset = 1 PSF; fit_psf: the same calibration with
 * kz_reset = 0.  Rows are ordered by frame, then by processing order; ids are
 * 0..n-1; frames are numbered from frame0.  Returns ZOLA_E_ARG with *nout set
 * to the needed size if out_cap is too small. */
ZOLA_API int zola_localize_frames(zola_ctx* ctx, zola_detector* det, zola_psf* fit_psf, const double* frames,
                                  int nframes, int frame0, const zola_loc_params* prm, zola_localization* out,
                                  int out_cap, int* nout);

/* Camera-count form of the pipeline: uint16 frames converted on the device
 * with adu, gain and offset exactly as zola_detect_u16 does
 * (LocalizationPipeline.java:100-107, 601-605); rows as zola_localize_frames. */
ZOLA_API int zola_localize_frames_u16(zola_ctx* ctx, zola_detector* det, zola_psf* fit_psf, const uint16_t* frames,
                                      int nframes, int frame0, const zola_loc_params* prm, double adu, double gain,
                                      double offset, zola_localization* out, int out_cap, int* nout);

/* sCMOS form of the pipeline (LocalizationPipeline.java:588-640, 799-820,
 * utils/SCMOScamera.java): adu frames (float, nframes x SX x SY) and per-pixel
 * offset, gain and variance maps (SX x SY).  Detection runs on
 * (adu - offset)/gain + vargain[0] clamped at 0, fits on (adu - offset)/gain +
 * vargain with vargain = variance / gain^2 added to the model mean; getAandB
 * works on patch - vargain. */
ZOLA_API int zola_localize_frames_scmos(zola_ctx* ctx, zola_detector* det, zola_psf* fit_psf, const float* adu,
                                        int nframes, int frame0, const zola_loc_params* prm, const double* offset,
                                        const double* gain, const double* variance, zola_localization* out,
                                        int out_cap, int* nout);

/* ThunderStorm-style CSV writer (data/PLocalization.java:224-306,
 * data/StackLocalization.java:1332-1360): header id,frame,x [nm],...,
 * occurrenceMerging; values floored to 1e-3 and printed as Java's
 * Double.toString; drift columns 0.0, occurrence 1.  append = 1 skips the header. */
ZOLA_API int zola_write_csv(const char* path, const zola_localization* locs, int n, int append);
/* Java Double.toString formatting of one value (the CSV number format). */
ZOLA_API int zola_format_double_java(double v, char* buf, int len);

/* --- Zernike calibration from bead z-stacks (replaces ZernikePhaseRetrieval's
 * stack NLL and its coordinate-wise finite-difference updates;
 * process/cpu/ZernikePhaseRetrieval.java:225-300, 860-1198, 1519-1530,
 * 1843-1874).  Bead b, slice s: PSF at (x_b, y_b, zoil = dz[s] + z_b,
 * zwat = 0) with phase sum_{i>=3} zernike[i] Z_i (modes 0-2, the reference's
 * per-bead registration, are carried as x_b, y_b, z_b and ignored in zernike)
 * and blur width sigma (px);
 *   mu = psi (photons[b][s] + a_bs) + sum_k c_bk m_k(i, ii),
 *   m = 1, i, i^2, ii, i ii, ii^2 (patch pixel (i, ii), first index x),
 * floored at 1e-8 as the reference; NLL = sum mu - d ln mu, FP64 on the GPU.
 * a_bs is the reference's fit_a + fit_a_each; c_bk its PolynomialBackground. */
typedef struct {
    int R;                 /* patch side (even) */
    int nz;                /* Zernike modes (4..231) */
    int nbead, nslice;
    const double* dz;      /* nslice slice offsets, um */
    const double* stacks;  /* nbead x nslice x R x R photons */
    const double* photons; /* nbead x nslice photon curve (zola_calib_init); NULL = 0 */
} zola_calib_data;
/* bead parameters per bead: x, y, z (um), a[nslice], c[6] */
#define ZOLA_CALIB_BEAD_STRIDE(nslice) (3 + (nslice) + 6)
ZOLA_API int zola_calib_forward(zola_psf* psf, const zola_calib_data* data, const double* zernike, double sigma,
                                const double* bead, double* nll,
                                double* model /* nullable: nbead x nslice x R x R */);
/* NLL and its exact gradient by the hand-written adjoint: grad_zernike[nz]
 * (0 for modes 0-2), grad_sigma (nullable), grad_bead (bead layout). */
ZOLA_API int zola_calib_backward(zola_psf* psf, const zola_calib_data* data, const double* zernike, double sigma,
                                 const double* bead, double* nll, double* grad_zernike, double* grad_sigma,
                                 double* grad_bead);
/* Levenberg-Marquardt fit of zernike[3..nz), sigma (with ZOLA_CALIB_FIT_SIGMA)
 * and every bead's parameters, updated in place: adjoint gradient,
 * Gauss-Newton matrix from device tangents, FP64 damped solve. */
#define ZOLA_CALIB_FIT_SIGMA 1
ZOLA_API int zola_calib_fit(zola_psf* psf, const zola_calib_data* data, double* zernike, double* sigma, double* bead,
                            int max_iter, int flags, double* nll, int* iters);
/* InitBackgroundAndPhotonNumber (process/InitBackgroundAndPhotonNumber.java:
 * 50-72, 110-420, 587-900): converts the raw stack (nslice x W x H, first
 * index x, ADU) to photons + 1 with slope adu/gain and offset, refines the
 * bead seeds (xpoints/ypoints, pixels, in place), fits the order-2 background
 * surface of the stack's low voxels, and returns per bead the background
 * background[nbead], the photon curve photons[nbead x nslice] (box-filtered
 * over +-max((int)(0.5/zstep)/2, 1) slices) and the patches
 * patches[nbead x nslice x size_patch^2] (outside the image: background).
 * poly_background (nullable) receives the W x H surface. */
ZOLA_API int zola_calib_init(zola_ctx* ctx, const float* raw, int nslice, int W, int H, float* xpoints,
                             float* ypoints, int nbead, int size_patch, double adu, double gain, double offset,
                             double zstep, double* photons, double* background, double* patches,
                             double* poly_background);

/* --- 3-D drift correction (replaces DriftCorrection / DriftCorrection_:
 * process/cpu/DriftCorrection.java:125-990, utils/SplineFit.java).
 * Localizations (x, y, z nm, frame; crlb nm, -1 or NULL = unknown) are binned
 * in time; all pairs of bins are cross-correlated as 3-D histograms in
 * half-overlapping windows of sizeFFT voxels (sizeFFT = the power of two
 * covering max_drift_um, the voxel grown by 1% steps until sizeFFT <= 128);
 * bin drifts relative to bin 0 come from the least squares over all pairs
 * (two passes of outlier rejection at the mean CRLB), and each localization's
 * drift from the spline of the bin drifts at its frame.
 * bin_drift: bins x (frame index, dx, dy, dz nm); loc_drift (nullable): n x 3
 * nm; pixel_nm_used (nullable): the voxel size after the growth. */
typedef struct {
    double pixel_nm;      /* histogram voxel (reference: pixelsizeNM) */
    int bins;             /* time bins */
    double max_drift_um;  /* subImageSizeUm: the window covers this drift */
} zola_drift_params;
ZOLA_API int zola_drift(zola_ctx* ctx, const double* xyz_nm, const double* crlb_nm, const int* frame, int n,
                        const zola_drift_params* prm, double* bin_drift, double* loc_drift, double* pixel_nm_used);

/* Allocation-free FP64 fit (this entry point has no counterpart in the
 * reference).  For callers that must not allocate device memory while they fit
 * (a host application that owns all device memory and lends plugins only its
 * own buffers; an acquisition thread that cannot stall on cudaMalloc/cudaFree,
 * which may synchronise the device): the plain FP64 fit of zola_fit_batch_dev
 * with its work areas and ROI counter in a 64 MiB array inside the library
 * image, held on every GPU that loads the library until the process exits.
 * Device buffers and stream as in zola_fit_batch_dev; prm->precision must be
 * ZOLA_PREC_FP64.  The PSF's tables for this ROI size must exist (any model or
 * fit call with this R, e.g. zola_psf_model_dev(psf, R, NULL, 0, NULL, NULL, s),
 * prepares them); the call itself allocates nothing.  It makes the PSF's
 * device current, as the other entry points do.  Its first call on a device
 * (and its first call after that device's context was destroyed and created
 * again, e.g. by cudaDeviceReset) looks up the array's device address; make
 * that first call before any stream capture.  ROI sizes whose per-block work area exceeds the array are
 * rejected with ZOLA_E_ARG; large windows run on fewer blocks.  All calls share
 * the array: calls that overlap on the GPU race, so serialise them. */
ZOLA_API int zola_fit_batch_noalloc(zola_psf* psf, int R, const float* d_rois, const double* d_init5, int n,
                                    const zola_fit_params* prm, double* d_out5, double* d_crlb5, double* d_nll,
                                    int* d_status, int* d_iters, void* stream);

/* Upper bound on the split fit's slot pool (ROIs in flight); 0 = automatic
 * (pool state up to 8 GB, at most 32768 slots).  Larger pools amortise each
 * launch's fixed work and shorten the draining tail of a batch. */
ZOLA_API int zola_ctx_set_pool(zola_ctx* ctx, int max_slots);
/* Split fit kernel layout.  ZOLA_SPLIT_STAGED (default) runs the five stages
 * (pupil DFT, window DFT, row blur, column blur + likelihood sums, FP64 LM
 * step) as five kernels per LM round over the whole slot pool.
 * ZOLA_SPLIT_FLOW runs the same stage code as one cooperative kernel: the
 * stages run at once on their own SMs, each unit of slots moves to the next
 * stage as soon as it is done, converged fits retire and refill from a device
 * queue, and there is no host round trip (the same results bit for bit; it
 * also takes inputs that are still arriving, zola_fit_batch_stream_dev).
 * ZOLA_SPLIT_FUSED runs stage 1 plus one kernel for stages 2-5 per round (same
 * arithmetic, FP32 sums in another order); windows whose fused plan does not
 * fit in shared memory run staged. */
#define ZOLA_SPLIT_STAGED 0
#define ZOLA_SPLIT_FUSED 1
#define ZOLA_SPLIT_FLOW 2
ZOLA_API int zola_ctx_set_split_mode(zola_ctx* ctx, int mode);
/* Dataflow kernel shape: units = units of slots in flight (0: two per SM),
 * ctas[5] = CTAs per stage (null or all 0: a split by window size; otherwise
 * each at least 1, adding up to the SM count).  Results do not depend on either. */
ZOLA_API int zola_ctx_set_flow(zola_ctx* ctx, int units, const int* ctas);
/* Autotuner of the dataflow kernel (enable = 1): the first large fits of each
 * class (pupil grid, ROI side) try a few shapes (CTAs per stage rebalanced
 * from each stage's measured busy time; 1.5, 2 and 3 units per SM) and keep the
 * fastest in device time per model evaluation.  Tuned shapes are read from and
 * written to cache_path (JSON, nullable).  A fit's results do not depend on the
 * shape, so tuning changes timings only. */
ZOLA_API int zola_ctx_set_tuning(zola_ctx* ctx, int enable, const char* cache_path);
/* Shape the dataflow kernel uses for psf's fits of R x R ROIs: units, ctas[5]
 * and, when tuned, the measured ns per model evaluation (nullable pointers).
 * Returns 1 when tuned, 0 for the default shape, < 0 on error. */
ZOLA_API int zola_fit_flow_shape(zola_psf* psf, int R, int* units, int* ctas, double* ns_per_eval);
/* The round-based split fit issues its kernels in blocks of four LM rounds (20
 * launches with the same arguments for the whole fit); enable = 1 (default)
 * captures a block once per fit as a CUDA graph and replays it, 0 launches
 * the kernels one by one.  Results are the same either way. */
ZOLA_API int zola_ctx_set_round_graphs(zola_ctx* ctx, int enable);
/* Slot pool of the round-based split fit (ZOLA_SPLIT_STAGED) for psf's R x R
 * ROIs.  With tuning on (zola_ctx_set_tuning) and no explicit pool
 * (zola_ctx_set_pool 0), the first four fits of a class with at least 131072
 * ROIs try pools of 4096, 8192, 16384 and 32768 slots (each capped at 8 GB of
 * pool state) and keep the fastest in device time per model evaluation; the
 * choice goes to the tuning cache file with the dataflow shapes, and mixed
 * batches use it too.  Returns 1 and the tuned pool (and its ns per
 * evaluation) when tuned, 0 and the context's setting (0: automatic) when not.
 * A fit's results do not depend on the pool. */
ZOLA_API int zola_fit_split_pool(zola_psf* psf, int R, int* pool, double* ns_per_eval);
/* Bookkeeping of the last dataflow fit on this context, per stage (pupil DFT,
 * window DFT, row blur, column blur + sums, LM step): the fraction of time its
 * CTAs had a unit to work on, and the busy GPU clocks one CTA spent per unit;
 * and the model evaluations made (nullable pointers, 5 values each). */
ZOLA_API int zola_ctx_flow_stats(zola_ctx* ctx, double* busy, double* clocks_per_unit, double* evaluations);
/* Upper bound, in GPU clocks, on the dataflow kernel's waits for a unit to
 * become ready (its schedulers and LM warps; e.g. for inputs still arriving);
 * 0 restores the default (2^31, about a second).  The mbarrier waits on bulk
 * copies and MMA completions keep a fixed bound of 2^31 clocks: a shorter one
 * could give up on a copy still in flight.  A wait that runs out ends the call
 * with ZOLA_E_TIMEOUT and leaves the context usable. */
ZOLA_API int zola_ctx_set_wait_limit(zola_ctx* ctx, long long clocks);

/* ---- CRLB curves and the z-centre search ------------------------------- */
/* Cramer-Rao bounds (x, y, z, A, B) of an emitter at (0, 0, z[i]) (um), zoil =
 * optics.zfocus, for n depths, from the finite-difference Fisher matrix of
 * process/cpu/CRLB.java:255-340 (computeFisher): central steps h (um) in x, y,
 * z; mu = photons psi + background; the A row steps the formed mean by +-a_step
 * photons (dmu/dA = mu a_step / h, as the reference) and the B row by +-h.
 * R is the model side (the reference uses the FFT grid size).  Replaces the
 * per-depth Java loops of CRLB.run (:73-160).  crlb5 is n x 5 (host). */
ZOLA_API int zola_crlb_curve(zola_psf* psf, int R, const double* z, int n, double photons, double background,
                             double h, double a_step, double* crlb5);
/* SearchPSFcenter.getPosition (process/cpu/SearchPSFcenter.java:37-84): the
 * depth z (um) that the localization pipeline stores as ZfocusCenter and
 * centres its [minZ, maxZ] = ZfocusCenter -+ axialRange / 2 on
 * (process/cpu/LocalizationPipeline.java:157-172).  Variant ZOLA_CENTER_CPU
 * follows process/cpu/SearchPSFcenter.java (h = 5 nm, A step 100 h);
 * ZOLA_CENTER_GPU follows process/gpu/SearchPSFcenter_.java (h = 0.5 nm, A step
 * h, and zfocus at once when n_oil == n_wat).  3000 photons, background 50, as
 * the reference.  axial_range <= 0 returns optics.zfocus.  R as above (the
 * reference builds its model at the FFT size, SearchPSFcenter.java:31). */
#define ZOLA_CENTER_CPU 0
#define ZOLA_CENTER_GPU 1
ZOLA_API int zola_psf_center_search(zola_psf* psf, int R, double axial_range, int variant, double* z_center);

/* Per-kernel timing.  With profiling on, every kernel launch of a fit or model
 * call is bracketed by CUDA events on its stream and the elapsed device time is
 * accumulated per kernel kind: 0..3 the split stages (pupil DFT, window DFT,
 * row blur, column blur with likelihood sums; the model-only column blur), 4
 * the fused stages 2-5, 5 the FP64 fit, 6 the FP64 model, 7 the split fit's LM
 * step and other kernels, 8 the dataflow split fit, 9 detection.
 * zola_ctx_stage_stats copies ZOLA_NSTAGES millisecond totals and launch
 * counts (either pointer may be null). */
#define ZOLA_NSTAGES 10
ZOLA_API int zola_ctx_profile(zola_ctx* ctx, int enable);
ZOLA_API int zola_ctx_stage_stats(zola_ctx* ctx, double* ms, long long* launches, int reset);

/* Number of kernel launches the library issued since the context was created
 * (bench bookkeeping). */
ZOLA_API long long zola_ctx_launches(const zola_ctx* ctx);

#ifdef __cplusplus
}
#endif
#endif /* ZOLA_B200_H */
