/* ertm_b200 — C ABI of the B200-native ERTM reverse-time-migration hot path.
 *
 * The reference (Sherlyn7189/Challenge-Cup) is a Python/NumPy package; its
 * hot path is ertm/propagation.py, ertm/imaging.py and ertm/numerics.py.  A
 * Python host binds this ABI with ctypes (challenge-cup_b200/ertm_b200/_lib.py)
 * and keeps the reference's call signatures; any other host can bind the
 * same symbols.  Each entry point below names the reference interface it
 * replaces.
 *
 * Conventions
 *  - Every function returns 0 on success and a negative code on failure;
 *    ertm_last_error() gives the message of the calling thread's last error.
 *  - Array arguments may be host or device pointers (unified addressing);
 *    copies use cudaMemcpyDefault.  Arrays are C-order float32 unless stated.
 *  - "padded" arrays have the reference geometry (nz+2·pad, nx+2·pad) with
 *    pad = order/2 + 1 (numerics.py:60-62, propagation.py:206-208).
 *  - A propagator owns one CUDA stream-ordered set of device buffers; all its
 *    work is enqueued on the stream given at creation (0 = legacy default).
 */
#ifndef ERTM_B200_H
#define ERTM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ERTM_OK 0
#define ERTM_ERR_ARG (-1)
#define ERTM_ERR_CUDA (-2)
#define ERTM_ERR_STATE (-3)
/* a wavefield became non-finite (NaN or infinity) during a run: an unstable
 * or overflowing propagation; other shots of a batch are unaffected */
#define ERTM_ERR_NONFINITE (-4)
/* propagator status bits (ertm_prop_status) */
#define ERTM_STATUS_NONFINITE 1u

/* engines (propagation.py:986-1001) */
#define ERTM_ENGINE_ACOUSTIC 0
#define ERTM_ENGINE_ELASTIC 1
#define ERTM_ENGINE_VISCO 2
/* boundaries (propagation.py:64-65) */
#define ERTM_BOUNDARY_CPML 0
#define ERTM_BOUNDARY_FREE 1
#define ERTM_BOUNDARY_NONE 2
/* record components */
#define ERTM_COMP_P 0
#define ERTM_COMP_VX 1
#define ERTM_COMP_VZ 2
#define ERTM_COMP_SXX 3
#define ERTM_COMP_SZZ 4
#define ERTM_COMP_SXZ 5
/* source mechanisms (types.py:137-159) */
#define ERTM_MECH_EXPLOSIVE 0
#define ERTM_MECH_SHEAR 1
#define ERTM_MECH_FORCE_Z 2
/* imaging conditions (imaging.py:61-87) */
#define ERTM_COND_ZERO_LAG 0
#define ERTM_COND_NORMALIZED 1
#define ERTM_COND_EXCITATION 2
/* wave types and P/S separation (imaging.py:47-52, propagation.py:945-977) */
#define ERTM_WAVE_P 0
#define ERTM_WAVE_S 1
#define ERTM_SEP_STRESS 0
#define ERTM_SEP_DIVCURL 1
/* imaging accumulators */
#define ERTM_ACCUM_FP64 0
#define ERTM_ACCUM_KAHAN 1

typedef struct ertm_prop_config {
  int32_t engine;            /* ERTM_ENGINE_* */
  int32_t order;             /* 2, 4, 6 or 8 */
  int32_t nx, nz;            /* physical grid */
  double dx, dz, x0, z0;     /* spacing and origin (types.py:20-82) */
  double dt;                 /* time step */
  int32_t free_surface;      /* 1: zero the free-surface row (acoustic p; elastic szz, sxz) */
  int32_t npml_x_left, npml_x_right, npml_z_top, npml_z_bottom; /* CPML strip widths, 0 = none */
  int32_t n_mech;            /* viscoacoustic: relaxation mechanisms L */
  int32_t n_q;               /* viscoacoustic: distinct Q values in the tables */
  int32_t compensation;      /* viscoacoustic: apply the amplitude cap / low-pass after each step */
  double amplitude_cap;      /* QOptions.amplitude_cap */
  int32_t lowpass_interval;  /* QOptions.lowpass_interval */
  int32_t reserved;
} ertm_prop_config;

typedef struct ertm_prop_info {
  int32_t nzp, nxp, ld, pad;
  int64_t state_bytes;       /* device bytes of one checkpoint (fields + CPML strips) */
  int64_t field_bytes;       /* reference field bytes (n_fields · nzp · nxp · 4) */
  int64_t step_index;
  int32_t n_fields, clipped, lowpass_steps, n_receivers;
  int32_t fast_div_x, fast_div_z;  /* 1: division by dx / dz uses the verified fast form */
  int32_t tile_rows, reserved;
} ertm_prop_info;

typedef struct ertm_migrate_config {
  int32_t nt;                /* len(wavelet): forward and replay steps */
  int32_t nt_spec;           /* spec.nt: excitation backward loop end (imaging.py:286-288) */
  int32_t interval;          /* checkpoint interval (imaging.py:121-124) */
  int32_t condition;         /* ERTM_COND_* */
  int32_t illumination;      /* bit 0: accumulate S² (normalized + illumination);
                                bit 1: accumulate R² (receiver normalisation) */
  int32_t start_step;        /* cross-correlation starts here (imaging.py:268-277) */
  int32_t separation;        /* ERTM_SEP_* (elastic) */
  int32_t n_images;          /* 1..2 images sharing one forward/replay/backward pass */
  int32_t src_wave[4];       /* ERTM_WAVE_* per image */
  int32_t rcv_wave[4];
  int32_t accum;             /* ERTM_ACCUM_* (excitation is always FP64) */
  int32_t n_comp;            /* record components */
  int32_t comp[8];           /* ERTM_COMP_* injection target per component (imaging.py:437-444) */
} ertm_migrate_config;

/* library ---------------------------------------------------------------- */
const char* ertm_last_error(void);
int32_t ertm_version(void);
/* Select the device and check it is sm_100 (no reference counterpart). */
int32_t ertm_init(int32_t device);
/* Instrumentation (no reference counterpart): kernels launched so far, and
 * CUDA-event timing of the stencil launches of every `every`-th step (or
 * batched tick) on the stream they run on; ertm_profile_read returns the
 * summed milliseconds, the number of timed samples and the algorithmic HBM
 * bytes of the timed launches since the last ertm_profile_stencil call. */
int64_t ertm_launch_count(void);
/* Pin the stencil tile height (8, 16 or 32 rows; 0 = automatic) for
 * propagators created afterwards — the autotuner's knob (order 8 only). */
int32_t ertm_set_tile_rows(int32_t rows);
/* Interior tiles (clear of CPML strips, free surface and source) in launches
 * of their own, apart from the boundary tiles: 0 = when the interior tiles
 * alone fill the GPU (default), 1 = never, 2 = whenever there are any.  The
 * results are the same either way; the knob is for tuning and tests. */
int32_t ertm_set_tile_split(int32_t mode);
/* Batched ticks: the works of a large (engine, order) group in one lane or
 * taken in turn by two or four lanes on separate streams (0 = automatic: two
 * when the group has at least 4 works and enough tiles, or the autotuner's
 * choice of one or two).  Results are identical. */
int32_t ertm_set_tick_lanes(int32_t lanes);
/* With two lanes: 0 alternates works between them (a shot's replay step on
 * one, its backward step on the other), 1 alternates shots (both steps of a
 * shot on one lane).  Results do not depend on it. */
int32_t ertm_set_lane_assign(int32_t mode);
/* Tile height of the boundary-frame launches when interior tiles run in
 * launches of their own: 0 the interior's, 8 or 16 rows (used when lower than
 * the interior's).  Results do not depend on it. */
int32_t ertm_set_frame_rows(int32_t rows);
/* Threads per CTA of the FFT line transforms of the wavenumber low-pass (a
 * multiple of 32 in [64, 1024]; 0 = chosen per transform length).  Results do
 * not depend on it. */
int32_t ertm_set_line_threads(int32_t threads);
/* 2, 4 or 8 (1 = 8): the elastic velocity phase of 32-row interior
 * rectangles marches down column strips in segments of at most that many
 * 16-row chunks (next chunk's copies in flight, z-halo rows in a ring)
 * instead of one block per tile (default 4); 0: tiles.  Results do not depend
 * on it. */
int32_t ertm_set_march(int32_t enable);
/* 1: the elastic stress phase of those interiors marches too, in the same
 * segments, with the fused imaging epilogue run per 16-row chunk; 0
 * (default): tiles.  Takes effect while ertm_set_march is non-zero.  Results
 * do not depend on it. */
int32_t ertm_set_march_stress(int32_t enable);
/* Online autotuning of batched ticks (default on): the first ticks of each
 * group shape (engine, order, works, size class) try tile heights 8/16/32,
 * split off/on and one or two lanes, timed with CUDA events; the fastest is
 * kept for the process.  Any forced knob above disables it.  1 = on, 0 = off,
 * −1 = off and forget the choices made so far.  Results do not depend on it. */
int32_t ertm_set_autotune(int32_t enable);
/* Interior tiles staged by TMA tiled bulk copies (1) or by cp.async (0, the
 * default: faster on the measured workloads).  Applies to propagators created
 * afterwards (their tensor maps are encoded at creation).  Results are
 * identical. */
int32_t ertm_set_tma(int32_t enable);
/* Bounded TMA waits that ran out since the library was loaded (0 in a healthy
 * run; −1 if the counter cannot be read).  A block whose wait runs out skips
 * its tile, so any non-zero value means wrong results. */
int64_t ertm_stage_timeouts(void);
/* One line per tuned group: each candidate tile height / split / lanes with
 * its mean tick time; the chosen one is starred.  Valid until the next call. */
const char* ertm_autotune_report(void);
/* Count, over all 2^32 float inputs a, where the fast division form `mode`
 * (3 one-FMA, 2 FMA correction, 1 float64 product) differs in value from
 * __fdiv_rn(a, h) (no reference counterpart; diagnostics). */
int32_t ertm_division_check(float h, int32_t mode, uint64_t* mismatches);
int32_t ertm_profile_stencil(int32_t enable, int32_t every);
int32_t ertm_profile_read(double* total_ms, int64_t* samples, double* total_bytes);

/* propagators ------------------------------------------------------------ */
/* Replaces AcousticPropagator/ViscoacousticPropagator/ElasticPropagator
 * construction (propagation.py:411-421, 518-606, 858-871): materials are
 * edge-padded and averaged on the device.  vp, vs, rho are physical (nz, nx).
 * The pml_a and pml_b arrays are the float32 CPML profiles (numerics.py:143-219) of the
 * padded axes.  The viscoacoustic tables (qidx, tau, delta, mref, relax_a)
 * come from the host-side GSLS fit (propagation.py:563-675); NULL otherwise. */
void* ertm_prop_create(const ertm_prop_config* cfg, const float* vp, const float* vs, const float* rho,
                       const float* pml_ax, const float* pml_bx, const float* pml_az, const float* pml_bz,
                       const uint8_t* qidx, const double* tau, const double* delta, const double* mref,
                       const float* relax_a, void* stream);
void ertm_prop_destroy(void* prop);
int32_t ertm_prop_info_get(void* prop, ertm_prop_info* info);
/* Propagator2D.reset (propagation.py:309-311, 423-428); clears the status word. */
int32_t ertm_prop_reset(void* prop);
/* Status word of a propagator (ERTM_STATUS_* bits), read after its queued
 * work: the stress phase sets ERTM_STATUS_NONFINITE when it writes NaN or
 * infinity.  No reference counterpart (the reference lets such a run finish
 * with a non-finite image); the checks follow the finite-value contracts of
 * types.py:106-122, 202-236 on the run's outputs. */
int32_t ertm_prop_status(void* prop, uint32_t* status);
/* Propagator2D.set_source (propagation.py:264-267): padded node and mechanism. */
int32_t ertm_prop_set_source(void* prop, int32_t iz, int32_t ix, int32_t mechanism);
/* Propagator2D.set_receivers (propagation.py:269-271): physical coordinates. */
int32_t ertm_prop_set_receivers(void* prop, int32_t n, const double* x, const double* z);
/* Propagator2D.step (propagation.py:314-316, 430-454, 686-723, 840-883):
 * n_steps steps with source amplitudes amps[0..n_steps) (host float64 array,
 * NULL = 0): the field receives float32(amp), the viscoacoustic strain
 * float32(amp / K_R) (propagation.py:707-713). */
int32_t ertm_prop_step(void* prop, int32_t n_steps, const double* amps);
/* Propagator2D.sample (propagation.py:456-470, 885-898): out is n_comp × nrec. */
int32_t ertm_prop_sample(void* prop, int32_t n_comp, const int32_t* comps, float* out);
/* Propagator2D.inject (propagation.py:472-494, 764-774, 900-942). */
int32_t ertm_prop_inject(void* prop, int32_t comp, const float* values);
/* Propagator2D.image_fields (propagation.py:500-501, 795-796, 945-977): (nz, nx). */
int32_t ertm_prop_image_field(void* prop, int32_t wave, int32_t separation, float* out);
/* Field / CPML-memory access for state()/load_state() (propagation.py:283-306).
 * Fields are padded (nzp, nxp); psi terms are expanded to full padded size. */
int32_t ertm_prop_read_field(void* prop, int32_t slot, float* out);
int32_t ertm_prop_write_field(void* prop, int32_t slot, const float* in);
int32_t ertm_prop_read_psi(void* prop, int32_t axis, int32_t term, float* out);
int32_t ertm_prop_write_psi(void* prop, int32_t axis, int32_t term, const float* in);
int32_t ertm_prop_set_step_index(void* prop, int64_t step_index);
/* Raw device checkpoint of the whole state block (state_bytes bytes). */
int32_t ertm_prop_save_state(void* prop, void* dst);
int32_t ertm_prop_load_state(void* prop, const void* src);

/* whole-loop drivers ------------------------------------------------------ */
/* run_forward (propagation.py:1018-1052): steps with amps[t] and samples the
 * components after each step into out (n_comp × nt × nrec). */
int32_t ertm_forward(void* prop, int32_t nt, const float* amps, int32_t n_comp, const int32_t* comps,
                     float* out);
/* RTMImager.migrate core (imaging.py:255-331): checkpointed forward,
 * block replay, time-reversed injection, backward propagation and the
 * imaging condition.  record is n_comp × nt_spec × nrec float32; the
 * accumulators are n_images × (nz, nx) float64 (num, illum, rillum). */
int32_t ertm_migrate(void* fwd, void* back, const ertm_migrate_config* cfg, const float* wavelet,
                     const float* record, double* num, double* illum, double* rillum);
/* One shot of a batched migration. */
typedef struct ertm_batch_shot {
  void* fwd;                 /* forward/replay propagator of this shot */
  void* back;                /* backward propagator of this shot */
  ertm_migrate_config cfg;
  const float* wavelet;      /* cfg.nt samples */
  const float* record;       /* cfg.n_comp × cfg.nt_spec × nrec */
  double* num;               /* outputs as in ertm_migrate */
  double* illum;
  double* rillum;
} ertm_batch_shot;

/* Batched form of ertm_migrate (the pipeline's shot loop, pipeline.py:277-283):
 * all shots advance together in ticks that share one velocity and one stress
 * launch per (engine, order) group; within a shot the replay of block b−1
 * overlaps the backward pass over block b.  Shots may differ in grid, engine,
 * length and condition.  Results equal n_shots separate ertm_migrate calls. */
int32_t ertm_migrate_batch(int32_t n_shots, const ertm_batch_shot* shots);

/* Batch sessions: the tick loop of ertm_migrate_batch made resumable, for a
 * serving loop (no single reference counterpart: it runs RTMImager.migrate,
 * imaging.py:205-349, for shots that join and leave between ticks).
 * ertm_session_add copies the shot's wavelet and record and prepares its
 * checkpoints; the shot's num/illum/rillum outputs must stay valid until
 * ertm_session_advance reports its tag done.  ertm_session_advance runs at
 * most max_ticks ticks, stopping early after the tick in which a shot
 * finishes, then writes the finished shots' accumulators and returns up to cap
 * of their tags.  A shot's propagators belong to the session until then. */
int32_t ertm_session_create(void** session);
int32_t ertm_session_add(void* session, const ertm_batch_shot* shot, int64_t tag);
int32_t ertm_session_advance(void* session, int32_t max_ticks, int64_t* done_tags, int32_t cap, int32_t* n_done);
int32_t ertm_session_active(void* session);
int64_t ertm_session_ticks(void* session);
int32_t ertm_session_destroy(void* session);
/* Shots of a session whose wavefields became non-finite: each advance checks
 * every active shot's propagators and takes such shots out of the session
 * (their accumulators are not finished); this returns and forgets up to cap
 * of their tags.  The other shots keep running. */
int32_t ertm_session_take_failed(void* session, int64_t* tags, int32_t cap, int32_t* n);

/* lowpass_wavenumber (numerics.py:424-442): out = Re(ifft2(fft2(in) · taper))
 * of an (nz, nx) float64 array, the radial taper 1 − (k − cutoff)/0.15
 * clipped to [0, 1] over the Nyquist-normalised wavenumbers.  The transforms
 * reproduce numpy.fft's arithmetic, so the result equals the reference's bit
 * for bit.  Host or device pointers; in place allowed. */
int32_t ertm_lowpass_wavenumber(int32_t nz, int32_t nx, double dx, double dz, double cutoff, const double* in,
                                double* out, void* stream);

/* Normalisation and _postprocess (imaging.py:326-333, 476-502): image =
 * num/(illum+eps)/(rillum+eps) as selected, Laplacian, wavenumber low-pass
 * (lowpass < 1), PML mask of width npml (top too when top_mask). */
int32_t ertm_postprocess(int32_t nz, int32_t nx, double dx, double dz, const double* num, const double* illum,
                         const double* rillum, int32_t by_illum, int32_t by_rillum, double eps,
                         int32_t laplacian, double lowpass, int32_t npml, int32_t top_mask, float* out,
                         void* stream);
/* Record preprocessing on the device (preprocess.py:36-224), for (nt, ntr)
 * float32 records, time-major; host or device pointers; float64 arithmetic
 * and one float32 rounding, as the reference.
 *   ertm_resample: Kaiser-windowed sinc resampling (numerics.py:337-392) with
 *     the host-computed weights w (n_out × taps) and first tap offsets off0
 *     (n_out; clamped to the record): out[o,s] = Σ_t w[o,t]·in[off0[o]+t, s].
 *   ertm_mute: direct-wave mute (preprocess.py:121-173), per-receiver ramp
 *     bounds start/end (seconds) at sample times t.
 *   ertm_taper: cosine end taper (preprocess.py:176-191) with the w-sample ramp.
 *   ertm_rotate: COG→CSG rotation of (vx, vz) by cos/sin (preprocess.py:36-67). */
int32_t ertm_resample(const float* in, int64_t n_in, int64_t ntr, const double* w, const int64_t* off0, int32_t taps,
                      int64_t n_out, float* out, void* stream);
int32_t ertm_mute(const float* in, int64_t nt, int64_t ntr, const double* t, const double* start, const double* end,
                  float* out, void* stream);
int32_t ertm_taper(const float* in, int64_t nt, int64_t ntr, const double* ramp, int64_t w, float* out,
                   void* stream);
int32_t ertm_rotate(const float* vx, const float* vz, int64_t n, double c, double s, float* ox, float* oz,
                    void* stream);

/* Time-varying filter (qcomp.py:98-147): S Hann-windowed frames of L samples
 * every hop samples of the (n, ntr) float64 record, each frame's spectrum
 * (L/2+1 frequencies) times its complex response (S × (L/2+1) interleaved
 * re/im float64), inverse, windowed overlap-add in frame order, divided by
 * the summed squared window.  Host or device pointers; out is (n, ntr)
 * float64. */
int32_t ertm_stft_filter(const double* in, int64_t n, int64_t ntr, int32_t L, int32_t hop, int32_t S,
                         const double* window, const double* response, double* out, void* stream);

/* SEG-Y rev 1 trace samples, replacing segyio's trace reads and writes in
 * segy.py:103-155 (read_segy_shots, read_segy_image) and segy.py:373-530
 * (write_segy_shot/shots/image).  A trace block is 240 header bytes followed
 * by ns big-endian samples, format 1 (IBM hex float) or 5 (IEEE float).
 *
 * decode: traces is the trace section (n_traces blocks of 240 + 4·ns bytes,
 * 4-byte aligned; host or device).  Output column c reads trace order[c] and
 * writes its samples to out[dest[c] + s·width[c]], s < ns, so one call fills
 * every shot's (ns, nrec) record of a file in its grouped, sorted order.
 * order/dest/width are host arrays (ncols each), checked against n_traces and
 * out_len (float32 elements) before the launch; out is host or device.
 *
 * encode: rec is (ns, ntr) float32; headers is ntr·240 bytes, big-endian,
 * copied unchanged; traces receives the ntr trace blocks. */
int32_t ertm_segy_decode(const uint8_t* traces, int64_t n_traces, int64_t ns, int32_t fmt, int64_t ncols,
                         const int32_t* order, const int64_t* dest, const int32_t* width, float* out,
                         int64_t out_len, void* stream);
int32_t ertm_segy_encode(const float* rec, int64_t ns, int64_t ntr, int32_t fmt, const uint8_t* headers,
                         uint8_t* traces, void* stream);

/* stack_images (pipeline.py:133-161): images is n_images pointers to (n,)
 * float32, each host or device memory (device images are read in place, host
 * images uploaded in groups of at most 1 GiB); out is host or device memory.
 * All images of a group go through two launches: every image's max|.|, then
 * the float64 sum over the images in order at each pixel. */
int32_t ertm_stack(int32_t n_images, int64_t n, const float* const* images, int32_t normalize, float* out,
                   void* stream);

/* pipeline.py:143-151 split in two so the sum can cross GPUs: the float64
 * accumulation loop (per image: max|.| when normalize, divide, add in image
 * order) and the final divide + cast.  ertm_stack_partial adds the images into
 * sum (a caller-zeroed device array of n float64, kept across calls); images
 * may be host or device pointers.  ertm_stack_finish writes
 * out = float32(sum / count) (device arrays).  A one-image stack is the image
 * itself in the reference, so callers pass normalize = 0 when the whole stack
 * holds one image. */
int32_t ertm_stack_partial(int32_t n_images, int64_t n, const float* const* images, int32_t normalize, double* sum,
                           void* stream);
int32_t ertm_stack_finish(int64_t n, const double* sum, int64_t count, float* out, void* stream);

/* No counterpart in the reference.  Same result as ertm_stack, but it
 * allocates nothing, for callers that cannot allocate device memory: a
 * serving process that carves all device memory into its own pool at start-up,
 * a host framework that owns every allocation, or code that must avoid the
 * device-wide synchronisation cudaMalloc/cudaFree may cause.  images (a host
 * array of n_images device pointers) and out must be device memory; more
 * than 1024 images per call is rejected with an error.  Scratch lives in
 * static device arrays (2 MiB of float64 sums + 4 KiB), held by every GPU that
 * loads the library until the process exits; the first call on a device looks
 * up their addresses (cudaGetSymbolAddress), so make that first call before any
 * stream capture.  Work is enqueued on `stream`; calls that overlap on the GPU
 * share the scratch and race, so order them on one stream. */
int32_t ertm_stack_noalloc(int32_t n_images, int64_t n, const float* const* images, int32_t normalize, float* out,
                           void* stream);

#ifdef __cplusplus
}
#endif

#endif /* ERTM_B200_H */
