/*
 * emc_b200.h -- C-ABI of the B200-native orientation-search hot path.
 *
 * Every entry point takes plain pointers, sizes and an explicit CUDA stream
 * (passed as void*; NULL = legacy default stream).  Device buffers are owned
 * by the caller; the library allocates only inside the opaque handles made by
 * the *_create / *_plan functions and frees it in the matching *_destroy.
 * No C++ exception crosses this boundary: every function returns emc_status.
 *
 * Conventions shared by all volume functions (they follow the reference):
 *   - volumes are x-fastest, linear index (z*ny + y)*nx + x
 *     (reference mexFiles/mexXform3d.cu:86);
 *   - the rotation origin is floor(n/2) on every axis (mexXform3d.cu:49-51);
 *   - 3x3 matrices are column-major (MATLAB order), as mexXform3d reads them
 *     (mexXform3d.cu:170-172);
 *   - half spectra are (nx/2+1) x ny x nz interleaved complex float, FFT order,
 *     the cuFFT/MATLAB R2C layout the reference's mexFFT returns
 *     (mexFiles/mexFFT.cu:96-131).
 */
#ifndef EMC_B200_H
#define EMC_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define EMC_API __attribute__((visibility("default")))
#else
#define EMC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef int emc_status;
#define EMC_OK             0
#define EMC_E_ARG         -1   /* bad argument (size, null pointer, unsupported combination) */
#define EMC_E_CUDA        -2   /* a CUDA runtime call failed; see emc_last_error() */
#define EMC_E_OOM         -3   /* device allocation inside a handle failed */
#define EMC_E_TIMEOUT     -4   /* a bounded device-side wait gave up */
#define EMC_E_UNSUPPORTED -5   /* size / mode not compiled into this library */

/* Human-readable text of a status and the last error message of the calling thread. */
EMC_API const char* emc_status_string(emc_status s);
EMC_API const char* emc_last_error(void);
/* Library version string and the compiled FFT edge lengths (for callers that pad). */
EMC_API const char* emc_version(void);

/* ------------------------------------------------------------------------ */
/* Rotation matrices and search grids (host, FP64)                          */
/* ------------------------------------------------------------------------ */

/* BH_defineMatrix(angles, 'Bah', direction) (coordinates/BH_defineMatrix.m:85-126).
 * direction: 0 = 'forward' (angles negated), 1 = 'inv' (order reversed).
 * R_out: 9 doubles, column-major. */
EMC_API emc_status emc_define_matrix(const double angles_deg[3], int direction, double R_out[9]);

/* eulerSearch(symmetry, theta_max, theta_step, psi_max, psi_step, ...) grid
 * (coordinates/eulerSearch.m:38-177), enumerated in the order the alignment
 * loop walks it (alignment/BH_alignRaw3d_v2.m:1119-1170: theta, then phi, then
 * psi).  Each orientation is the triple (phi, theta, psi) in degrees, the
 * rotation passed on is defineMatrix([phi, theta, psi - phi], 'inv').
 * Call once with out = NULL to get *count, then again with room for 3*count.
 * symmetry: "C<n>", "D<n>", "O", "I", "I2". theta_max < 0 selects the
 * bipolar search of the reference. */
EMC_API emc_status emc_euler_search(const char* symmetry, double theta_max, double theta_step,
                            double psi_max, double psi_step,
                            double* out_phi_theta_psi, int* count);

/* ------------------------------------------------------------------------ */
/* mexXform3d: rotate + shift + interpolate a volume                        */
/*   replaces mexFiles/mexXform3d.cu:93-324 (create / reuse / destroy) and   */
/*   the testScripts/interpolator.m handle class (:29-154, :401-408)         */
/* ------------------------------------------------------------------------ */

typedef struct emc_volume_s* emc_volume_t;

#define EMC_INTERP_LINEAR   0   /* trilinear, interpn(...,'linear',0) semantics: 0 outside [0,n-1] */
#define EMC_INTERP_CUBIC    1   /* tricubic (Catmull-Rom), 0 outside the volume */
#define EMC_INTERP_LINEAR_BORDER 2 /* trilinear with zero-valued border voxels, the texture
                                      cudaAddressModeBorder behaviour of mexXform3d.cu:269-271,
                                      evaluated with FP32 weights */

#define EMC_DTYPE_F32  0
#define EMC_DTYPE_BF16 1

/* Copies the source volume (nx*ny*nz floats, device) into a handle-owned
 * buffer, optionally stored as bf16 (FP32 interpolation either way). */
EMC_API emc_status emc_xform3d_create(const float* d_src, int nx, int ny, int nz, int store_dtype,
                              emc_volume_t* out, void* stream);
/* out[p] = (1/nsym) * sum_s I(M_s (p - c + sh) + c)   with
 *   fwd != 0 ('forward'): sh = -shift, applied before the rotation
 *   fwd == 0 ('inv')    : the shift is added after the rotation
 * (mexXform3d.cu:45-65, :160-168).  R: nsym column-major 3x3 matrices (FP64,
 * rounded to FP32 as the reference does).  d_out: nx*ny*nz floats. */
EMC_API emc_status emc_xform3d_apply(emc_volume_t h, const double* R, int nsym, const float shift[3],
                             int fwd, int interp, float* d_out, void* stream);
EMC_API emc_status emc_xform3d_destroy(emc_volume_t h);

/* ------------------------------------------------------------------------ */
/* mexFFT: R2C / C2R 1-, 2- and 3-D transforms, unnormalised                */
/*   replaces mexFiles/mexFFT.cu:16-239 and fourierTransformer.m:38-159      */
/* ------------------------------------------------------------------------ */

typedef struct emc_fft_s* emc_fft_t;

/* dims: logical real sizes {nx, ny, nz} (x fastest; unused trailing dims = 1).
 * Every dim > 1 must be 2^a 3^b and <= 512.  batch >= 1 volumes back to back. */
EMC_API emc_status emc_fft_plan(int rank, const int dims[3], int batch, emc_fft_t* out);
/* d_in: nx*ny*nz floats per batch item; d_out: (nx/2+1)*ny*nz complex (float2). */
EMC_API emc_status emc_fft_r2c(emc_fft_t p, const float* d_in, float* d_out_complex, void* stream);
/* inverse of the above, unnormalised (like cufftExecC2R); d_in is not modified. */
EMC_API emc_status emc_fft_c2r(emc_fft_t p, const float* d_in_complex, float* d_out, void* stream);
EMC_API emc_status emc_fft_destroy(emc_fft_t p);

/* ------------------------------------------------------------------------ */
/* mexCTF / mexSF3D                                                          */
/* ------------------------------------------------------------------------ */

typedef struct {
  float pixel_size;     /* Angstrom */
  float wavelength;     /* Angstrom */
  float cs_mm;          /* spherical aberration, mm */
  float amp_contrast;   /* amplitude contrast fraction (converted to a phase, core_headers.cuh:71-72) */
  float defocus1;       /* Angstrom, positive = underfocus */
  float defocus2;       /* Angstrom */
  float astig_deg;      /* astigmatism angle, degrees from x */
} emc_ctf_params;

/* mexCTF(half, sq, nX, nY, pix, lambda, Cs, df1, df2, ast, AC[, centred])
 * (mexFiles/mexCTF.cu:6-121, kernel mexFiles/utils/ctf.cu:12-66).
 * d_out: (half ? nx/2+1 : nx) * ny floats. */
EMC_API emc_status emc_ctf2d(const emc_ctf_params* p, int nx, int ny, int half, int squared, int centred,
                     float* d_out, void* stream);
/* The exposure-filtered variant (mexFiles/utils/ctf.cu:68-130). */
EMC_API emc_status emc_ctf2d_exposure(const emc_ctf_params* p, int nx, int ny, int half, int squared,
                              int centred, float radial_weight, float total_exposure,
                              float* d_out, void* stream);
/* mexSF3D(half, sq, size[3], pix[n], lambda[n], Cs[n], df1[n], df2[n], ast[n], AC[n],
 *         nTilts, tilt[n], exposure[n], occupancy[n]) (mexFiles/mexSF3D.cu:84-302):
 * sum over tilts of the exposure-weighted CTF^2 inserted on the tilted central
 * slab.  Host arrays of n_tilts entries; d_out: size[0]*size[1]*size[2] floats,
 * overwritten.  half must be 0 (the reference only builds the full grid). */
EMC_API emc_status emc_sf3d(int half, int squared, const unsigned size[3], const float* pix,
                    const float* wavelength, const float* cs_mm, const float* df1,
                    const float* df2, const float* astig_deg, const float* amp_contrast,
                    unsigned n_tilts, const float* tilt_deg, const float* exposure,
                    const float* occupancy, float* d_out, void* stream);

/* Per-particle Fourier weight on the half spectrum ((n/2+1)*n*n floats, FFT order): the
 * binary Y-tilt-axis missing wedge of BH_weightMask3d 'binaryWedge' (masking/BH_weightMask3d.m:
 * 103-120; cones of +/-(90-|tilt|) around kz removed, |kx|,|kz| <= 2 slab kept, times the
 * 'nyquist' window of BH_bandpass3d; the Gaussian smoothing of :124-131 is not applied) times,
 * when ctf != NULL, the CTF
 * of the 3-D spatial frequency (mexFiles/utils/ctf.cu:45-62; defocus1 used, no astigmatism),
 * squared when squared != 0. */
EMC_API emc_status emc_wedge_ctf_weight(int n, float tilt_min_deg, float tilt_max_deg, const emc_ctf_params* ctf,
                                        int squared, float* d_out, void* stream);

/* BH_weightMask3d(SIZE, tilts, 'binaryWedgeGPU', ..) (masking/BH_weightMask3d.m:99-143) for a Y tilt
 * axis: the binary wedge on the centred n^3 grid (theta = atan2d(X, Z); the cones of
 * +/-(90 - |tilt|) removed; the |X|, |Z| <= 2 slab kept), smoothed (smooth != 0) by convn with
 * BH_multi_gaussian3d(9, 1.5) ('same', zero outside), times the 'nyquist' window of BH_bandpass3d,
 * then (W - min) / max(W - min).  layout 0: the centred n^3 volume the reference returns; layout 1:
 * its ifftshifted half spectrum ((n/2+1)*n*n, FFT order), the form the search takes as wdgMask.
 * Scratch (two n^3 volumes) comes from the stream-ordered allocator. */
EMC_API emc_status emc_binary_wedge(int n, float tilt_min_deg, float tilt_max_deg, int smooth, int layout,
                                    float* d_out, void* stream);
/* EMC_maskShape('sphere', SIZE, RADIUS, 'gpu', {'shift', shift; 'kernel', kernel_frac})
 * (masking/EMC_maskShape.m:95-224): the ellipsoid of radius RADIUS + ceil(k/2) centred at
 * floor(SIZE/2) + shift (single-precision test, as MATLAB), the outer ceil(k/2) voxels of every
 * face zeroed, blurred by the separable Gaussian of k = max(9, round((min(SIZE) kernel_frac - 1)/2)*2+1)
 * taps and sigma = sqrt(-(ceil(k/2)/2)^2 / (2 ln 0.5)), divided by its maximum, values <= 0.001 set
 * to 0.  kernel_frac = 0.04 is the reference's default; 0 gives the binary ellipsoid.  size[2] == 1
 * makes a 2-D mask.  shift may be NULL.  d_out: size[0]*size[1]*size[2] floats, x fastest. */
EMC_API emc_status emc_mask_sphere(const int size[3], const double radius[3], const double shift[3],
                                   double kernel_frac, float* d_out, void* stream);
/* BH_multi_cRef(fscINFO, radialGrid, bFactor, flgAlignRef) (statistics/BH_multi_cRef.m:1-166; the
 * isotropic filter, cones being off there): F = the not-a-knot cubic spline through (shell_freq,
 * max(shell_fsc, 0)); cRef = the not-a-knot spline through (os_freq, sqrt(|2F/(1+F)|) .* MTF .*
 * force_mask) with the ad hoc MTF of fscINFO{3}{3} (0: none; 1, 2 and other values as the
 * reference); the filter is cRef(|k| / pixel_size) on the half spectrum (FFT order) of a
 * size[0] x size[1] x size[2] volume, the particle bandpass of BH_alignRaw3d_v2.m:524-531.
 * Frequencies in 1/Angstrom; force_mask may be NULL (= 1).  Synchronises the stream. */
EMC_API emc_status emc_cref_filter(const double* shell_freq, const double* shell_fsc, int n_shells,
                                   const double* os_freq, const double* force_mask, int n_os, double mtf,
                                   const int size[3], float pixel_size, float* d_out, void* stream);

/* ------------------------------------------------------------------------ */
/* Volume and spectrum operators around the search                          */
/* ------------------------------------------------------------------------ */

/* BH_padZeros3d(IMAGE, padLow, padTop, 'GPU', 'single'|'singleTaper', fill)
 * (masking/BH_padZeros3d.m:79-229): negative pads trim, positive pads add `fill`; taper != 0
 * blends the 7 outermost voxels of every face towards `fill` with 0.5+0.5cos((0:6)pi/7).
 * d_out: (nx+pl+pt) x ... floats. */
EMC_API emc_status emc_pad3d(const float* d_in, int nx, int ny, int nz, const int pad_low[3], const int pad_top[3],
                             float fill, int taper, float* d_out, void* stream);
/* BH_bandpass3d(SIZE, HIGH_THRESH, HIGH_CUT, LOW_CUT, 'GPU', PIXEL_SIZE) (masking/BH_bandpass3d.m:
 * 54-170) on the half spectrum (FFT order).  pixel_size > 0: cut-offs in Angstrom; pixel_size == 0:
 * 'nyquist'; pixel_size < 0: 'nyquistHigh'. */
EMC_API emc_status emc_bandpass3d(int nx, int ny, int nz, float high_thresh, float high_cut, float low_cut,
                                  float pixel_size, float* d_out, void* stream);
/* BH_bandLimitCenterNormalize(IMG, BANDPASS, [], PAD, 'single'|'singleTaper')
 * (masking/BH_bandLimitCenterNormalize.m:40-61): pad with the image mean, fftn, F(0) = 0, times the
 * bandpass (half spectrum or NULL), F / (sqrt(sum |F|^2) / numel).  Output: half spectrum. */
EMC_API emc_status emc_band_limit_center_normalize(const float* d_img, int nx, int ny, int nz,
                                                   const int pad_low[3], const int pad_top[3], int taper,
                                                   const float* d_bandpass, float* d_spectrum_out,
                                                   void* stream);
/* BH_multi_xcf_Rotational(rotPART_FT, REF_FT, wdgMask, refWdg) (statistics/BH_multi_xcf_Rotational.m:
 * 71-78), unweighted form: sum Re(refWdg P R wdgMask) / sqrt(sum |R wdgMask|^2 sum |P refWdg|^2) over
 * the full spectrum; R is the already-conjugated reference spectrum; weights may be NULL (= 1). */
EMC_API emc_status emc_xcf_rotational(const float* d_part_ft, const float* d_ref_ft_conj, const float* d_wdg_mask,
                                      const float* d_ref_wdg, int nx, int ny, int nz, double* h_cc,
                                      void* stream);
/* BH_multi_xcf_Translational(A, B, peakMask, peakCOM) (statistics/BH_multi_xcf_Translational.m:31-104):
 * map = fftshift(real(ifftn(A .* B))), peakMask < 0.95 set to the map minimum, argmax (first index),
 * two centre-of-mass passes on the (2 peakCOM + 1)^3 box of map - min, peak minus the origin.
 * peak_mask (fftshifted, n^3) may be NULL; d_map_out (optional) receives the fftshifted map. */
EMC_API emc_status emc_xcf_translational(const float* d_a, const float* d_b, int nx, int ny, int nz,
                                         const float* d_peak_mask, int peak_com, double peak_out[3],
                                         double* max_val, float* d_map_out, void* stream);

/* ------------------------------------------------------------------------ */
/* Fused orientation search (BH_alignRaw3d_v2.m:1119-1423 inner body,        */
/* BH_multi_xcf_Translational_2.m:35-38 normalised CC,                        */
/* BH_multi_xcf_Translational.m:31-42 masked argmax)                          */
/* ------------------------------------------------------------------------ */

typedef struct emc_search_s* emc_search_t;

/* Particle side of one search item.  The search scores every orientation with the normalised
 * translational CC of BH_multi_xcf_Translational_2.m:35-38,
 *   map = real(ifftn(refWdg .* rotPART_FT .* REF_FT .* wdgMask)) * numel
 *         / sqrt(sum |REF_FT .* wdgMask|^2 * sum |rotPART_FT .* refWdg|^2),
 * with REF_FT = conj(wref .* fftn(rotated, masked reference)), DC = 0.  The particle's operands are
 *   spectrum = refWdg .* rotPART_FT, rotPART_FT = B .* F(particle) with F(0) = 0
 *              (BH_bandLimitCenterNormalize.m:48-55), as emc_particle_spectrum makes it with
 *              weight = refWdg;  energy = sum |spectrum|^2;
 *   wedge    = wdgMask, a real half spectrum that multiplies the rotated reference's spectrum (NULL
 *              = 1).  With BH_multi_xcf_Rotational's binding (BH_alignRaw3d_v2.m:1376-1383: the
 *              particle's wedge on the reference, the reference's wedge on the particle) this is
 *              the particle's own missing-wedge / CTF weight and refWdg is the reference's. */
typedef struct {
  const float* spectrum;   /* device, (n/2+1)*n*n complex */
  double energy;           /* sum over the full spectrum of |spectrum|^2 */
  double prior[9];         /* column-major R_prior (BH_alignRaw3d_v2.m:1176) */
  float  shift[3];         /* estPeakCoord applied with the reference rotation */
  int    box;              /* n: 64, 96 or 128 */
  int    ref_id;           /* reference registered with emc_search_add_reference */
  int    orient_begin;     /* slice [begin, begin+count) of the orientation list */
  int    orient_count;
  const float* wedge;      /* device, (n/2+1)*n*n floats (FFT order), or NULL */
} emc_particle_desc;

typedef struct {
  float cc;                /* normalised CC at the peak */
  int   orient;            /* orientation index (global index into the list) */
  int   peak[3];           /* integer peak shift (x, y, z) relative to the origin */
} emc_search_hit;

/* Q = weight .* bandpass .* fftn(particle) with Q(0) = 0; *energy = sum |Q|^2 over the
 * full spectrum (Hermitian-weighted, FP64).  weight/bandpass: real half spectra
 * (n/2+1)*n*n in FFT order, either may be NULL (= 1).  d_energy: one device double.
 * For the search, weight is the CC formula's refWdg (the weight that multiplies the particle)
 * and bandpass the particle's bandpassFilt. */
EMC_API emc_status emc_particle_spectrum(int n, const float* d_particle, const float* d_weight,
                                 const float* d_bandpass, float* d_spectrum_out,
                                 double* d_energy, void* stream);
/* emc_particle_spectrum over `count` particles in one call (three FFT passes and one weighting
 * launch for the whole batch instead of five launches per particle): d_particles [count][n^3],
 * d_weights [count][(n/2+1)*n*n] or NULL, d_bandpass one shared half spectrum or NULL,
 * d_spectra_out [count][(n/2+1)*n*n] complex, d_energies [count].  The per-particle loop of
 * BH_alignRaw3d_v2.m:1089-1100 (particle weight, BH_bandLimitCenterNormalize) batched; each
 * particle's result equals emc_particle_spectrum's.  At most 65535 particles per call. */
EMC_API emc_status emc_particle_spectra(int n, int count, const float* d_particles,
                                const float* d_weights, const float* d_bandpass,
                                float* d_spectra_out, double* d_energies, void* stream);

EMC_API emc_status emc_search_create(emc_search_t* out);
/* Registers a reference volume (n^3 floats, device), an optional real-space mask
 * applied after rotation (n^3, or NULL) and an optional real half-spectrum weight
 * applied to the rotated reference's spectrum (bandpass; NULL = 1).  store_dtype:
 * EMC_DTYPE_F32 or EMC_DTYPE_BF16 (mixed precision: interpolation stays FP32). */
EMC_API emc_status emc_search_add_reference(emc_search_t s, const float* d_ref, int n,
                                    const float* d_mask, const float* d_wref,
                                    int store_dtype, int* ref_id, void* stream);
/* Orientation list: n triples (phi, theta, psi) in degrees; the search rotation of
 * particle p, orientation o is  RotMat = R_prior(p) * defineMatrix([phi,theta,psi-phi],'inv')
 * and the reference is sampled through RotMat' with 'forward' semantics
 * (BH_alignRaw3d_v2.m:1175-1176, :1287-1291).  Composition runs in FP64 on the device. */
EMC_API emc_status emc_search_set_orientations(emc_search_t s, const double* phi_theta_psi, int n);
/* Tuning knobs (0 = automatic / autotuned).  peak_radius: spherical peak mask radius in
 * voxels (the peakMask >= 0.95 region of BH_multi_xcf_Translational.m:34).  chunk_evals:
 * evaluations per launch of the three passes; 0 cuts each box's evaluations into equal chunks of
 * at most 768 MiB of scratch (about 520 evaluations at 64^3), or an eighth of the free device
 * memory at creation if less, and into at least two at 64^3 (whose chunks overlap in pairs). */
EMC_API emc_status emc_search_configure(emc_search_t s, int peak_radius, int interp, int chunk_evals);
/* Runs every (particle, orientation) pair.  d_cc / d_peak (optional, may be NULL):
 * per-pair outputs in pair order (particle-major, orientations in list order),
 * d_peak holds 3 ints per pair.  d_best: one hit per particle (stable argmax over its
 * orientations, first index wins ties, as sortrows(...,-6) at BH_alignRaw3d_v2.m:1423).
 * All outputs are device memory.  Uneven box sizes are allowed in one call; the
 * launch sequence is captured in a CUDA graph, and the graphs of the four most recent distinct
 * requests are kept and replayed when a request repeats (a double-buffered pipeline alternating
 * between two descriptor sets replays both). */
EMC_API emc_status emc_search_run(emc_search_t s, const emc_particle_desc* particles, int n_particles,
                          float* d_cc, int* d_peak, emc_search_hit* d_best, void* stream);
/* emc_search_run with the particle energies read on the device: d_energy[p] replaces
 * particles[p].energy (which is ignored) and is read when the run executes on the stream,
 * so spectra from emc_particle_spectrum can feed the search with no host round trip in
 * between.  No counterpart in the reference, where the energy is a MATLAB scalar computed
 * on the host per particle (BH_alignRaw3d_v2.m:1098-1100 via BH_bandLimitCenterNormalize);
 * a particle whose energy is not > 0 scores CC = 0. */
EMC_API emc_status emc_search_run_energies(emc_search_t s, const emc_particle_desc* particles,
                                   int n_particles, const double* d_energy, float* d_cc,
                                   int* d_peak, emc_search_hit* d_best, void* stream);
/* Same as emc_search_run with host output buffers (copies inside, synchronises).  The device
 * staging buffers stay in the handle between calls (grown on demand), so repeating a request
 * replays its recorded graph.  Returns EMC_E_TIMEOUT when a device-side wait of the run gave up
 * (see emc_search_status). */
EMC_API emc_status emc_search_run_host(emc_search_t s, const emc_particle_desc* particles,
                               int n_particles, float* h_cc, int* h_peak,
                               emc_search_hit* h_best, void* stream);
/* No counterpart in the reference.  Synchronises `stream` and reports whether a device-side wait of
 * the handle's runs since the last check gave up (EMC_E_TIMEOUT; the results of those runs are
 * invalid), clearing the report.  The waits (for the bulk copies of the z and peak passes) are bounded
 * at about a second, after which the CTA leaves without a result; the context stays usable. */
EMC_API emc_status emc_search_status(emc_search_t s, void* stream);
/* Test hook (no counterpart in the reference): waits of later runs give up after wait_cycles SM
 * clock cycles (default 2^31), and announce phantom_bytes (a multiple of 16, at most 4096) more
 * bytes than they copy, so that with phantom_bytes > 0 every such wait runs out.
 * emc_search_test_wait(s, 1ll << 31, 0) restores the defaults. */
EMC_API emc_status emc_search_test_wait(emc_search_t s, long long wait_cycles, unsigned phantom_bytes);
EMC_API emc_status emc_search_destroy(emc_search_t s);
/* Measurement hook (no counterpart in the reference).  With profiling enabled, emc_search_run
 * launches eagerly instead of through the graph and brackets each pass launch with CUDA events
 * on the calling stream.  emc_search_timings returns, summed over all runs since the last
 * reset, the device time in ms of pass A (rotate + xy R2C), pass B (z FFT, multiply, inverse z),
 * pass C (inverse xy + peak, and the decode of each evaluation by its last pass-C CTA) and a
 * fourth slot (the time between pass C's end and the chunk's end, now only event overhead),
 * their launch counts, and the number of CC evaluations.  launches_last_run: kernels launched by
 * the most recent run. */
EMC_API emc_status emc_search_set_profiling(emc_search_t s, int enable);
EMC_API emc_status emc_search_timings(emc_search_t s, double ms[4], long launches[4], long* evals,
                                      long* launches_last_run, int reset);

/* Tuning hook (no counterpart in the reference).  Pass A (rotate + xy R2C) runs planes = 1, 2, 4
 * or 8 z-planes per CTA.  Unless fixed here, the first emc_search_run that meets a (box, dtype)
 * times pass A on its first chunk with every planes value whose slab fits shared memory and
 * keeps the fastest for that handle.  emc_search_set_planes fixes the value for one box (both
 * dtypes; EMC_E_ARG if it does not divide the box or does not fit), 0 returns it to tuning.
 * emc_search_get_planes reports the value in use for (box, dtype), 0 if not tuned yet, and the
 * pass-A time of each option at tuning (ms_per_option[k] for planes = 1 << k, -1 where not
 * timed; may be NULL). */
EMC_API emc_status emc_search_set_planes(emc_search_t s, int box, int planes);
EMC_API emc_status emc_search_get_planes(emc_search_t s, int box, int dtype, int* planes, float ms_per_option[4]);
/* Tuning hook (no counterpart in the reference).  A recorded run keeps slots = 1 or 2 sets of chunk
 * scratch (2 by default); with 2, consecutive 64^3 chunks go to two branches of the CUDA graph and
 * run concurrently (the passes of one chunk fill the tails of the other's), chunks of one slot in
 * order; chunks of larger boxes always run one at a time.  Profiled runs
 * (emc_search_set_profiling) use one slot so that per-pass times stay separable. */
EMC_API emc_status emc_search_set_overlap(emc_search_t s, int slots);


/* Single-particle search that allocates no device memory.  No counterpart in the reference.
 * For callers that may not call cudaMalloc after start-up: hosts whose own pool owns the GPU
 * memory (MATLAB's gpuArray allocator, a framework caching allocator), where a raw allocation
 * can fail or fragment the pool, and loops that must keep a bounded latency.  All scratch lives
 * in one static 24 MiB device array per GPU, held until the process exits.  The first call on a
 * device resolves that array's address and uploads FFT twiddles on the caller's stream (make it
 * before any stream capture); under CUDA's default lazy module loading that first call is also
 * when the driver allocates the array, so make it (any valid small search) at start-up, before the
 * caller's pool takes the GPU's memory, or load modules eagerly (CUDA_MODULE_LOADING=EAGER).
 * Every call reuses the same array, so calls that overlap on the GPU race; the call synchronises
 * the stream before returning.  The search runs with no particle wedge (wdgMask = 1): fold any
 * particle-side weight into d_spectrum.  Limits (EMC_E_ARG beyond them): box 64, 96 or 128,
 * FP32 reference, 1..4096 orientations (host (phi, theta, psi) triples), peak radius 1..15.
 * Same arguments and outputs as emc_search_run for one particle (device outputs may be NULL);
 * EMC_E_TIMEOUT (results invalid) if a bounded device-side wait gave up, as emc_search_status. */
EMC_API emc_status emc_search_plain_noalloc(const float* d_ref, const float* d_mask, int n,
                                            const float* d_spectrum, double energy, const double prior[9],
                                            const float shift[3], const double* phi_theta_psi, int n_orient,
                                            int peak_radius, int interp, float* d_cc, int* d_peak,
                                            emc_search_hit* d_best, void* stream);

/* ------------------------------------------------------------------------ */
/* Forward + adjoint of the masked CC w.r.t. 3 Euler angles and 3 shifts      */
/* ------------------------------------------------------------------------ */

/* For each of n poses (phi, theta, psi in degrees; tx, ty, tz in voxels), evaluates
 *   CC = sum_p r(p) h(p) / sqrt(E_R E_P)
 * with r = mask .* I(M (p - c - t) + c) the rotated, shifted reference (tricubic),
 * M = (R_prior * defineMatrix([phi,theta,psi-phi],'inv'))', h = unnormalised
 * inverse transform of the particle spectrum and E_R the DC-free reference energy,
 * i.e. the zero-lag value of the normalised CC map of the search, and its exact
 * gradient (dCC/dphi, dtheta, dpsi per degree, dCC/dt per voxel).
 * h: n^3 floats (from emc_particle_template).  Outputs: h_cc[n], h_grad[6n] host. */
EMC_API emc_status emc_particle_template(int n, const float* d_spectrum, float* d_h, void* stream);
EMC_API emc_status emc_cc_adjoint(emc_search_t s, int ref_id, const float* d_h, double energy_p,
                          const double prior[9], const double* poses, int n_poses,
                          double* h_cc, double* h_grad, void* stream);
/* Batched form for many particles in one launch: item i uses reference ref_ids[i], template d_h[i]
 * (device pointer), energy energy_p[i], prior priors[9i..9i+8] and pose poses[6i..6i+5].
 * interp: EMC_INTERP_CUBIC (smooth, as emc_cc_adjoint) or EMC_INTERP_LINEAR (trilinear through the
 * reference's corner cells, one vector load per voxel; piecewise-linear objective). */
EMC_API emc_status emc_cc_adjoint_batch(emc_search_t s, int n_items, const int* ref_ids,
                                        const float* const* d_h, const double* energy_p, const double* priors,
                                        const double* poses, int interp, double* h_cc, double* h_grad,
                                        void* stream);

/* ------------------------------------------------------------------------ */
/* Template search (BH_templateSearch3d_2.m:633-887)                          */
/* ------------------------------------------------------------------------ */

typedef struct emc_tsearch_s* emc_tsearch_t;

/* Tomogram nx*ny*nz (device floats, already locally normalised), every dim 2^a 3^b <= 512.
 * The tomogram spectrum is computed once and multiplied by the swapQuadrants phase
 * ramp (BH_templateSearch3d_2.m:633-641, :714). */
EMC_API emc_status emc_tsearch_create(const float* d_tomo, int nx, int ny, int nz,
                              emc_tsearch_t* out, void* stream);
/* template: t^3 floats (device, t <= min dim), zero-padded into the centre of the volume
 * (BH_templateSearch3d_2.m:752); orientations as in emc_search_set_orientations but
 * the template is sampled with defineMatrix([phi,theta,psi-phi],'forward')
 * (:744).  For each orientation the CC map is divided by its standard deviation
 * (:764) and the per-voxel max and the 1-based index of the winning orientation are
 * kept (:851-854, strict '<' so the first orientation wins ties).  d_peak / d_angle:
 * nx*ny*nz floats, initialised by the call. */
EMC_API emc_status emc_tsearch_run(emc_tsearch_t h, const float* d_template, int t,
                           const double* phi_theta_psi, int n_orient,
                           float* d_peak, float* d_angle, void* stream);
EMC_API emc_status emc_tsearch_destroy(emc_tsearch_t h);

/* Template-search post-processing (BH_templateSearch3d_2.m:1100-1275, nPeaks = 1): greedy peak
 * picking on the (padded) score map d_mag (modified in place) with the angle-index map d_ang
 * (1-based indices into angle_list, <= 0 = none).  Repeats, while fewer than max_peaks peaks are
 * recorded, fewer than max_tries iterations were made and the map maximum exceeds high_thr:
 * take the first maximum; if its angle index is > 0, record
 * sampling * (c + centre of mass of the 3^3 box - rm_dim) (c 1-based), the angle_list row and the
 * maximum, and zero the (2 rm_dim + 1)^3 box where the removal mask (h_removal, that size, host),
 * rotated by the row's angles (defineMatrix(row, 'Bah', 'forward'), zero border), is >= mask_cutoff;
 * otherwise zero that voxel.  angle_list: n_angles x 3 (the [phi, theta, psi - phi] rows of
 * ANGLE_LIST).  h_peaks: max_peaks x 10 doubles (x, y, z, e1, e2, e3, 0, 0, 0, score), *n_found
 * rows filled (the reference then keeps rows with x > 0). */
EMC_API emc_status emc_tsearch_peaks(float* d_mag, const float* d_ang, int nx, int ny, int nz,
                                     const float* h_removal, int rm_dim, float mask_cutoff,
                                     const double* angle_list, int n_angles, int max_peaks, int max_tries,
                                     float high_thr, float sampling, double* h_peaks, int* n_found,
                                     void* stream);
/* BH_movingAverage_2(img, featureSize) (statistics/BH_movingAverage_2.m): separable Gaussian
 * moving average (length featureSize, sigma 3, symmetric boundaries). */
EMC_API emc_status emc_moving_average(const float* d_in, int nx, int ny, int nz, int feature_size,
                                      float* d_out, void* stream);
/* The local normalisation of BH_templateSearch3d_2.m:558-561, in place:
 * x <- (x - avg(x)) / sqrt(avg(x^2) - avg(x)^2) with avg = emc_moving_average. */
EMC_API emc_status emc_local_normalize(float* d_vol, int nx, int ny, int nz, int feature_size, void* stream);

/* ------------------------------------------------------------------------ */
/* Subtomogram averaging (transformations/BH_average3d.m:1207-1500)           */
/* ------------------------------------------------------------------------ */

/* Symmetry operators the interpolator applies for "C<n>", "D<n>" or "O"
 * (testScripts/interpolator.m:172-214), column-major 3x3 each, identity first.  For D<n> that is
 * the n in-plane rotations only: the reference stores the mirrored copies but never applies them
 * (nSymMats = n).  out may be NULL to query *count; at most 60 matrices. */
EMC_API emc_status emc_symmetry_matrices(const char* symmetry, double* out, int* count);

typedef struct emc_average_s* emc_average_t;

/* Running odd / even half-set sums of BH_average3d.  n: particle box; d_mask: the soft
 * interpolation mask interpMask (n^3, device; copied), whose voxels > bin_threshold (0.01 in the
 * reference, :1087-1092) form the statistics region; nw: box of the wedge / CTF weights (0: no
 * weights); sym / nsym: symmetry matrices (column-major, as emc_symmetry_matrices; NULL and 1 for
 * C1); batch: particles rotated per pass (0: sized for about 2 GB of scratch). */
EMC_API emc_status emc_average_create(int n, const float* d_mask, float bin_threshold, int nw,
                                      const double* sym, int nsym, int batch, emc_average_t* out,
                                      void* stream);
/* Adds particles, in order (:1417-1482).  d_particles: count extracted windows [count][n^3]
 * (device); rot: [count][9] host, the geometry's rotation matrix (columns 17:25, column-major);
 * shift: [count][3] host (NULL = 0), the subvoxel shift of the window; weight: [count] host
 * (peakWgt; NULL = 1); half: [count] host, 1 (ODD) or 2 (EVE).  Each particle is rotated with
 * interpolator(vol, rot, shift, 'inv', symmetry): s = (rot S_k)(p - c) + shift + c with a zero
 * border, averaged over k; normalised r = (r - mean(r(B))) / rms(r(B) - mean) .* mask; dropped
 * when mean(r(:)) is not finite; then r .* weight is added to its half set.  With wedges,
 * d_wedges holds n_wedges weight volumes [n_wedges][nw^3] (device) and wedge_index[p] picks the
 * particle's one, rotated the same way with a zero shift and added (times weight) when the
 * particle is kept.  kept (host, may be NULL): 1 for particles added, 0 for dropped ones.
 * Synchronises the stream. */
EMC_API emc_status emc_average_add(emc_average_t a, const float* d_particles, int count,
                                   const double* rot, const float* shift, const float* weight,
                                   const int* half, const float* d_wedges, int n_wedges,
                                   const int* wedge_index, int* kept, void* stream);
/* Half set `half` (1 or 2): d_avg (n^3, may be NULL) = sum / count (:1703-1707; NaN when the half
 * set is empty), d_wedge_sum (nw^3, may be NULL) = the summed rotated weights, *count (may be
 * NULL) = particles added. */
EMC_API emc_status emc_average_result(emc_average_t a, int half, float* d_avg, float* d_wedge_sum,
                                      long* count, void* stream);
EMC_API emc_status emc_average_reset(emc_average_t a, void* stream);
/* Particle box and wedge box (0: none) of a handle. */
EMC_API emc_status emc_average_boxes(emc_average_t a, int* n, int* nw);
EMC_API emc_status emc_average_destroy(emc_average_t a);

/* ifftshift of count centred volumes (nx*ny*nz each, x fastest) cropped to their half spectra
 * ((nx/2+1)*ny*nz each, FFT order): the weight volumes of the reference (SF3D, wedge masks; centred
 * as the reference builds them, then ifftshift-ed before use, e.g. iMaxWedgeIfft at
 * BH_alignRaw3d_v2.m:1092-1099) in the form the search reads as wdgMask.  Not in place. */
EMC_API emc_status emc_centred_to_half(const float* d_in, int nx, int ny, int nz, int count, float* d_out,
                                       void* stream);
/* BH_weightMaskMex(SIZE, SAMPLING, TLT, xyzSubTomo, reconGeometry) (masking/BH_weightMaskMex.m:1-60)
 * for count particles: the tilt table (rows x cols, row-major as emc_tlt_read; columns as
 * :16-30) is sorted on column 1 and cast to single; each particle's defocus is offset by the
 * height of its position along every tilt's beam; the volumes come from emc_sf3d (full grid, CTF
 * squared) and are shifted by -(min - 1e-4).  xyz: [count][3]; recon_geometry: the 2 x 3
 * reconGeometry, row-major (size, then shift); d_out: [count][size^3].  All particles' tilt images
 * are made by one launch per chunk of particles (under 1 GiB of images) and accumulated by a
 * second; the call synchronises the stream once. */
EMC_API emc_status emc_sf3d_particles(const unsigned size[3], double sampling, const double* tlt, int rows,
                                      int cols, const double* xyz, const double recon_geometry[6], int count,
                                      float* d_out, void* stream);

/* ------------------------------------------------------------------------ */
/* Data formats either side of the path: MRC volumes, tilt tables, windows   */
/* ------------------------------------------------------------------------ */

typedef struct {
  int nx, ny, nz, mode;      /* mode 0 (int8), 1 (int16), 2 (float32), 6 (uint16) are read */
  int mx, my, mz;            /* sampling (cell divisions) */
  float cell[3];             /* cell dimensions, Angstrom */
  float pixel_size[3];       /* cell / m */
  float dmin, dmax, dmean, rms;
  float origin[3];
  int ext_bytes;             /* extended header bytes */
  int imod_stamp, imod_flags;
  long data_offset;          /* 1024 + ext_bytes */
  int byte_swapped;          /* 1 when the file has the other byte order */
} emc_mrc_header;

/* The header words MRCImage reads (@MRCImage/private/readHeader.m:1-176), with its byte-order
 * detection (a negative or > 65535 size means the file is byte-swapped). */
EMC_API emc_status emc_mrc_read_header(const char* path, emc_mrc_header* out);
/* getVolume(mrc, [x1 x2], [y1 y2], [z1 z2]) (@MRCImage/getVolume.m:150-298): box = {x1, x2, y1,
 * y2, z1, z2}, 1-based inclusive, zeros (or box NULL) for a whole axis; converted to float (mode 0
 * read as signed int8, as getVolume does).  h_out: (x2-x1+1)(y2-y1+1)(z2-z1+1) floats, x fastest. */
EMC_API emc_status emc_mrc_read(const char* path, const int* box, float* h_out);
/* Same box straight into device memory: sections stream through two pinned staging buffers and are
 * converted to float on the GPU while the next block is read.  Synchronises the stream. */
EMC_API emc_status emc_mrc_read_device(const char* path, const int* box, float* d_out, void* stream);
/* SAVE_IMG(vol, name, pixelSize[, origin]) for float32 volumes (@MRCImage/SAVE_IMG.m): mode 2, cell =
 * n * pixel size, min / max / mean and the std(std(std(vol))) rms of SAVE_IMG in the header. */
EMC_API emc_status emc_mrc_write(const char* path, const float* h_vol, int nx, int ny, int nz,
                                 const float pixel_size[3], const float origin[3]);
/* A whitespace-separated numeric table such as <tilt>_ctf.tlt (columns per
 * masking/BH_weightMaskMex.m:16-30); out (may be NULL): rows x cols doubles, row-major. */
EMC_API emc_status emc_tlt_read(const char* path, double* out, int max_rows, int* rows, int* cols);
/* BH_isWindowValid(volumeSize, windowSize, maskRadius, center) (logicals/BH_isWindowValid.m):
 * start = 0-based volume index of window voxel 0 (the window holds vol(start + i), zero outside),
 * pad_low / pad_top = the zero padding, shift = center - floor(center), valid = 0 for 'noUse'
 * (available extent < 2 (maskRadius + 6) - 2 on some axis).  Output pointers may be NULL. */
EMC_API emc_status emc_window_bounds(const int volume_size[3], const int window_size[3], double mask_radius,
                                     const double center[3], int start[3], int pad_low[3], int pad_top[3],
                                     double shift[3], int* valid);
/* Extracts count windows (BH_average3d.m:1304-1341: crop + BH_padZeros3d with zeros) from a device
 * volume nx*ny*nz in one launch: d_out [count][wz][wy][wx]; centers [count][3] in the reference's
 * 1-based volume coordinates; shifts [count][3] and valid [count] (host, may be NULL) as
 * emc_window_bounds. */
EMC_API emc_status emc_extract_windows(const float* d_vol, int nx, int ny, int nz, const int window_size[3],
                                       const double* centers, int count, double mask_radius, float* d_out,
                                       double* shifts, int* valid, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* EMC_B200_H */
