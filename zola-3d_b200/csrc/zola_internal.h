// Internal types shared by the host set-up, the kernels and the C-ABI.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/zola_b200.h"

namespace zola {

// Per-PSF pupil tables on the disk's bounding square (D x D, row a <-> kx,
// column b <-> ky), zero outside the disk.  Built on the host in FP64 from
// the optics (process/PhaseParameters.java:300-362, process/cpu/PSFPhase.java:140-220).
struct PsfView {
    int N;          // pupil grid (power of two)
    int D;          // disk bounding-square side
    int a0;         // first disk row / column index in the N grid
    double dx;      // um
    double zfocus;  // zoil of the localization model, um
    const double* pupil;    // D*D amplitude (0 outside the disk)
    const double* phase;    // D*D Zernike phase, radians
    const double* kz;       // D*D
    const double* kzoil;    // D*D
    const double* isim;     // D*D (1: propagating in the sample)
    const double* isimoil;  // D*D
    const double* kx;       // D   (kx of row a)
    const double* ky;       // D   (ky of column b)
};

// Per-ROI-size tables: the partial-DFT twiddles and the circular blur.
struct WinView {
    int R;          // ROI side
    int W;          // intensity window, pow2(min(2R, N)) (PSFPhase.java:100-108)
    const double2* C;   // W x D: C[w][a] = exp(+2 pi i ((a0+a+N/2)(w-W/2) mod N) / N)
    const double* G;    // R x W: blur row i' <- window row i (circulant, see optics.cpp)
};

struct FitParamsDev {
    double zmin, zmax, xymax, tol_xyz, step_xy, step_z;
    int max_iter;
    // Likelihood resolution of the fit: a step whose predicted decrease is at
    // most this is accepted unless the likelihood rose by more than this (0:
    // a step is accepted only when the likelihood did not rise).
    double accept_nll = 0.0;
};

// The ROIs, start points and outputs of a fit.
struct FitIO {
    const float* rois;
    const float* scmos;  // sCMOS var/gain^2 per pixel (Localization.java:1132), or null
    const double* init;
    int n;
    FitParamsDev prm;
    double* out5;
    double* crlb5;
    double* nll;
    int* status;
    int* iters;
};

// Host-side tables of one window size (FP64 and the split-precision packs).
struct WindowTables {
    int R = 0, W = 0;
    std::vector<double> C;     // W*D*2 interleaved
    std::vector<double> G;     // R*W
    double2* d_C = nullptr;
    double* d_G = nullptr;
    // split-precision operand packs (tcgen05 path), built lazily
    void* d_split = nullptr;
    size_t split_bytes = 0;
};

}  // namespace zola

namespace zola {
// Shape of the dataflow split-fit kernel: units of slots in flight and CTAs per
// stage (pupil DFT, window DFT, row blur, column blur + sums, LM step).
constexpr int FLOW_STAGES = 5;
struct FlowShape {
    int units = 0;
    int ctas[FLOW_STAGES] = {0, 0, 0, 0, 0};
};
// Autotuning state of one (pupil grid, disk rows, ROI side, window) class: the
// trials made so far and the best shape measured, in device ns per model
// evaluation.
struct FlowTune {
    FlowShape best, next;
    double best_ns = 0;
    int trials = 0;
    bool done = false;
};
// Autotuning state of the round-based split fit of one class: the slot pool
// size, tried from small to large, kept by device ns per model evaluation.
struct PoolTune {
    int best = 0;
    double best_ns = 0;
    int trials = 0;
    bool done = false;
};
}  // namespace zola

struct zola_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t copy_stream = nullptr;    // host-to-device input copies that overlap the fit
    std::vector<cudaEvent_t> feed_ev;      // completion of each input chunk of a host-buffer fit
    std::string err;
    long long launches = 0;
    int num_sms = 0;
    // reusable device scratch (FP64 fit work areas, counters)
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    // grow-only device staging for the host-buffer entry points (inputs and
    // results of one call; never overlaps scratch)
    void* io = nullptr;
    size_t io_bytes = 0;
    void* calib_area = nullptr;  // calibration work buffers (grow-only, reused by every call)
    size_t calib_bytes = 0;
    void* calib_fit_area = nullptr;  // the calibration LM's tangents, Gram blocks and model (grow-only)
    size_t calib_fit_bytes = 0;
    int* d_counter = nullptr;
    int* d_status_word = nullptr;
    int* h_flags = nullptr;      // pinned host words read back by the split fit loop
    int split_pool_max = 0;      // 0: size the split slot pool automatically
    bool round_graphs = true;    // replay the round-based split kernels as CUDA graphs
    int split_mode = ZOLA_SPLIT_STAGED;  // ZOLA_SPLIT_STAGED, _FUSED or _FLOW
    int flow_units = 0;          // dataflow kernel: units of slots in flight (0: automatic)
    int flow_ctas[5] = {};       // dataflow kernel: CTAs per stage (all 0: automatic)
    long long wait_limit = 0;    // clocks a device wait may take before the call fails (0: about a second)
    cudaStream_t feed_stream = nullptr;  // copies of the arrived-ROI count of a host-buffer fit
    cudaEvent_t ev_init = nullptr;
    int* h_feed = nullptr;       // pinned chunk ends for those copies
    // dataflow-kernel autotuner: on (1) / off (0), JSON cache file, state per class
    int tune = 0;
    std::string tune_path;
    std::map<std::string, zola::FlowTune> tunes;
    std::map<std::string, zola::PoolTune> pool_tunes;
    cudaEvent_t tune_ev[2] = {nullptr, nullptr};
    unsigned long long* h_tune = nullptr;  // pinned: evaluations, then (idle, total clocks, units) per CTA
    double flow_busy[5] = {};              // last dataflow launch: busy fraction per stage
    double flow_clk_per_unit[5] = {};      // last dataflow launch: busy clocks per unit per stage (one CTA)
    double flow_evals = 0;                 // last dataflow launch: model evaluations
    // mixed batches: a stream and a read-back event per class (the last event
    // orders the classes after the caller's stream), pinned flag words
    cudaStream_t mix_stream[ZOLA_MAX_CLASSES] = {};
    cudaEvent_t mix_ev[ZOLA_MAX_CLASSES + 1] = {};
    int* h_mix = nullptr;
    // optional per-kernel timing with CUDA events on the launch stream
    int profile = 0;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<int> ev_stage;   // stage id of each recorded (start, stop) pair
    int ev_used = 0;
    double stage_ms[ZOLA_NSTAGES] = {};
    long long stage_launches[ZOLA_NSTAGES] = {};
};

namespace zola {
struct DetView {
    int SX, SY, R, Z, cap;
    double inv_m;        // 1 / sqrt(Mx My)
    double thr, zstep, dx;
    const double* psf0;  // Z x R x R zero-mean library PSFs
    const double* varpsf;
    const double* norm;  // SX x SY box counts (normImage)
};
}  // namespace zola

struct zola_detector {
    zola_psf* psf = nullptr;
    zola::DetView v{};
    std::vector<double> range;
    double* d_lib = nullptr;    // psf0 | varpsf | norm
    std::vector<double> h_psf;  // Z x R x R normalised library PSFs (pipeline initialisation)
    int cand_room = 0;          // longest candidate list the pipeline has met (its next starting room)
};

namespace zola {
// Kernel-timing helpers (capi.cu): bracket a launch when profiling is on.
void prof_begin(zola_ctx* ctx, int stage, cudaStream_t st);
void prof_end(zola_ctx* ctx, cudaStream_t st);
void prof_collect(zola_ctx* ctx);  // call after the stream was synchronised
}  // namespace zola

struct zola_psf {
    zola_ctx* ctx = nullptr;
    zola_optics o{};
    int N = 0, K = 0, D = 0, a0 = 0;
    std::vector<double> zern;
    // host copies of the D x D tables
    std::vector<double> pupil, phase, kz, kzoil, isim, isimoil, kx, ky;
    double* d_tables = nullptr;  // one allocation holding the arrays below
    zola::PsfView view{};
    std::map<int, zola::WindowTables> win;
};

namespace zola {

// optics.cpp
int build_psf_tables(zola_psf* p, const zola_optics* o, const double* zern, int nz, std::string& err);
int window_size(int R, int N);
WindowTables* get_window(zola_psf* p, int R, std::string& err);
void blur_matrix(int R, int W, double sigma, std::vector<double>& G, std::vector<double>* dG);

// fit_f64.cu
// d_list / d_count (nullable): evaluate only the models d_list[0 .. *d_count) (at most n).
int launch_model_f64(zola_ctx* ctx, zola_psf* p, WindowTables* w, const double* d_xyz, int n,
                     double* d_out, double* d_dout, cudaStream_t st, const int* d_list = nullptr,
                     const int* d_count = nullptr);
int launch_fit_f64(zola_ctx* ctx, zola_psf* p, WindowTables* w, const float* d_rois, const float* d_scmos,
                   const double* d_init, int n, const zola_fit_params* prm, double* d_out5, double* d_crlb5,
                   double* d_nll, int* d_status, int* d_iters, cudaStream_t st);

// fit_split.cu
int launch_model_split(zola_ctx* ctx, zola_psf* p, WindowTables* w, const double* d_xyz, int n, double* d_out,
                       double* d_dout, cudaStream_t st);
void free_split_plan(void* plan);
void tune_load(zola_ctx* ctx);  // read the autotuner's cache file (zola_ctx::tune_path)
bool flow_shape(zola_ctx* ctx, zola_psf* p, WindowTables* w, FlowShape* out, double* ns_per_eval);
// ROIs that reach the device while a split fit runs (host-buffer calls): chunk
// c holds ROIs [chunk_end[c - 1], chunk_end[c]) and is on the device once ev[c]
// has completed.  The slot pool refills only from ROIs that have arrived.
struct RoiFeed {
    int n_chunks = 0;
    const int* chunk_end = nullptr;
    const cudaEvent_t* ev = nullptr;
};
// One class of a mixed batch: its PSF, window tables and fit inputs/outputs.
struct MixedClass {
    zola_psf* p;
    WindowTables* w;
    FitIO F;
};
// feeds (nullable): per class, its input chunks still arriving (n_chunks 0: all on the device)
int launch_fit_split_mixed(zola_ctx* ctx, int nc, MixedClass* mc, cudaStream_t st,
                           const RoiFeed* feeds = nullptr);
// The round-based split fit's pool for psf's R x R ROIs: 1 and the tuned pool
// (and its ns per evaluation) when tuned, else 0 and the context's setting.
int split_pool_choice(zola_psf* p, WindowTables* w, int* pool, double* ns_per_eval);
int launch_fit_split(zola_ctx* ctx, zola_psf* p, WindowTables* w, const float* d_rois, const float* d_scmos,
                     const double* d_init, int n, const zola_fit_params* prm, double* d_out5, double* d_crlb5,
                     double* d_nll, int* d_status, int* d_iters, cudaStream_t st, const RoiFeed* feed = nullptr,
                     const int* d_avail = nullptr);

int ensure_scratch(zola_ctx* ctx, size_t bytes, std::string& err);
// camera counts -> photons (LocalizationPipeline.java:601-605): rescale = {adu / gain, -offset adu / gain}
void camera_rescale(double adu, double gain, double offset, double* rescale);
void rescale_u16(zola_ctx* ctx, const uint16_t* d_in, size_t n, const double* rescale, double* d_out,
                 cudaStream_t st);
int ensure_io(zola_ctx* ctx, size_t bytes);

// Owned device allocation released on scope exit (one-time host paths).
template <class T>
struct DevBuf {
    T* p = nullptr;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, n * sizeof(T)); }
};

}  // namespace zola

#define ZOLA_CUDA_CHECK(call, ctxp)                                                 \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess) {                                                    \
            (ctxp)->err = std::string(#call) + ": " + cudaGetErrorString(e_);       \
            return ZOLA_E_CUDA;                                                     \
        }                                                                           \
    } while (0)
