/*
 * aob200.h -- C ABI of the B200-native adaptive-optics hot path.
 *
 * One shared library (libaob200.so) exports these entry points.  They take
 * plain pointers and sizes, return an int status (AOB_OK = 0, AOB_ERR = 1)
 * and never throw; the message of the last failure on the calling thread is
 * available from aob_last_error().  Streams are passed as void* (a
 * cudaStream_t; NULL = the legacy default stream).  Host arrays are in the
 * reference's Fortran (column-major) order: element (x, y) of an n x n map
 * is at x + y*n.
 *
 * Each entry point names the reference interface it replaces (paths within
 * the reference project).  The Python package `aob200` binds exactly these
 * symbols with ctypes.
 */
#ifndef AOB200_H
#define AOB200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define AOB_OK 0
#define AOB_ERR 1

/* ---- library --------------------------------------------------------- */

/* Message of the last failed call on this thread ("" if none). */
const char *aob_last_error(void);
/* Library version string. */
const char *aob_version(void);
/* Number of CUDA devices visible (0 when none); never fails. */
int aob_device_count(void);
/* Device name (NUL-terminated, truncated to len) and SM count. */
int aob_device_name(int device, char *buf, int len, int *num_sms);
/* Copies between host and a device buffer owned by this library or the
 * caller (the carma array buffer protocol, python_module/carma/src/obj.hpp:32-76). */
int aob_memcpy_d2h(void *dst_host, const void *src_dev, size_t bytes, void *stream);
int aob_memcpy_h2d(void *dst_dev, const void *src_host, size_t bytes, void *stream);
/* aob_memcpy_h2d without the final wait: the copy is enqueued on the stream
 * and the call returns (host memory must stay unchanged until the stream has
 * reached the copy; pinned memory keeps it asynchronous).  No counterpart in
 * the reference, whose array copies complete before they return. */
int aob_memcpy_h2d_async(void *dst_dev, const void *src_host, size_t bytes, void *stream);
int aob_memcpy_d2d(void *dst_dev, const void *src_dev, size_t bytes, void *stream);
int aob_malloc(void **dev_ptr, size_t bytes, int device);
int aob_free(void *dev_ptr);
int aob_stream_sync(void *stream);
/* Fill a device float buffer with a value (CarmaObj::memset / reset). */
int aob_fill_f32(float *dev, size_t n, float value, void *stream);

/* ---- Shack-Hartmann sensor ------------------------------------------ *
 * Replaces SutraWfsSH (libsutra/src.cpp/sutra_wfs_sh.cpp) as created by
 * SutraSensors (sutra_sensors.cpp:25-135) and bound by
 * python_module/sutra/src/wfs_sh.cpp:41-148.                             */
typedef struct aob_sh aob_sh;

/* Constructor arguments of SutraWfsSH (sutra_wfs_sh.cpp:27-75). npup is the
 * side of the guide-star phase screen the sensor reads (p_geom._n); ntot >= nfft
 * (ntot > nfft: the field of view extended beyond the spot's FFT support). */
int aob_sh_create(aob_sh **out, int device, int nxsub, int nvalid, int npix, int nphase,
                  int nrebin, int nfft, int ntot, int npup, float pdiam, float nphot,
                  float nphot4imat);
int aob_sh_destroy(aob_sh *h);
/* SutraWfsSH::load_arrays (sutra_wfs_sh.cpp:308-331).  phasemap [nphase^2,
 * nvalid] (indexes into the npup x npup phase screen) and ttprojmat
 * [nphase^2, 2 nvalid], both column-major, are kept for aob_sh_slopes_geom
 * and may be NULL; kernel is accepted for interface parity.  binmap is
 * [nrebin^2, npix^2] indexes into the ntot x ntot image, offsets [nphase^2];
 * fluxPerSub, validsubsx, validsubsy, istart and jstart have nvalid entries.
 * hrmap (nfft^2 positions of the nfft x nfft spot in the ntot x ntot image) is
 * required when ntot != nfft (extended field of view) and may be NULL
 * otherwise. */
int aob_sh_load_arrays(aob_sh *h, const int32_t *phasemap, const int32_t *hrmap,
                       const int32_t *binmap, const float *offsets, const float *fluxPerSub,
                       const int32_t *validsubsx, const int32_t *validsubsy,
                       const int32_t *istart, const int32_t *jstart, const float *ttprojmat,
                       const float *kernel_c64);
/* SutraSensors::set_field_stop / SutraWfsSH::set_field_stop (sutra_sensors.cpp:
 * 223-229, sutra_wfs_sh.cpp:674-707): a focal-plane field stop of the full
 * pupil, mask n x n (fftshifted, as the reference's geometry gives it), n a
 * power of two in [8, 2048] and >= npup.  Each image then forms the field
 * pupil * exp(i phase) in the top-left corner of the n x n plane, multiplies
 * its FFT by the mask and reads the sub-aperture fields from the inverse FFT
 * (sutra_wfs_sh.cpp:366-391).  mask NULL or n == 0 removes it.  Steps with a
 * field stop run the separate-kernel path (not the fused RTC kernel or the
 * batch). */
int aob_sh_set_field_stop(aob_sh *h, const float *mask, int n);
/* fakecam (Sensors(..., fakecam, max_flux_per_pix, max_pix_value),
 * sutra_wfs_sh.cpp:95-105,623-643): every image is also digitised into the
 * uint16 frame "camimg", min((binimg * flat + dark) / max_flux_per_pix, 1) *
 * max_pix_value truncated (digitalize_krnl, libsutra/src.cu/sutra_wfs.cu:
 * 2243-2255); dark starts at 0 and flat at 1.  Steps with fakecam run the
 * separate-kernel path. */
int aob_sh_set_fakecam(aob_sh *h, int enable, int max_flux_per_pix, int max_pix_value);
/* Wfs.set_dark / set_flat (python_module/sutra/src/wfs.cpp) of the fakecam
 * digitisation: n x n with n the image side. */
int aob_sh_set_dark(aob_sh *h, const float *dark, int n);
int aob_sh_set_flat(aob_sh *h, const float *flat, int n);
/* SutraWfs::set_pupil (sutra_wfs.cpp) -- npup x npup amplitude. */
int aob_sh_set_pupil(aob_sh *h, const float *pupil_host);
/* SutraWfs::set_noise (sutra_wfs.cpp:123-141); the generator is the
 * project's Philox4x32-10 keyed by seed (not cuRAND). */
int aob_sh_set_noise(aob_sh *h, float noise, int64_t seed);
/* Guide-star wavelength in micron: phase scale 2*pi/lambda (sutra_source.cpp:97). */
int aob_sh_set_lambda(aob_sh *h, float lambda_um);
int aob_sh_set_nphot(aob_sh *h, float nphot);
/* Frame counter used as the noise-stream counter (advances on each noisy image). */
int aob_sh_set_frame(aob_sh *h, uint64_t frame);
int aob_sh_get_frame(aob_sh *h, uint64_t *frame);
/* Device pointers of the sensor's buffers (the Wfs d_* properties,
 * python_module/sutra/src/wfs.cpp:54-225). which: "phase", "pupil",
 * "bincube", "binimg", "intensities", "validsubsx", "validsubsy",
 * "fluxPerSub", "binmap", "offsets", "istart", "jstart", "slopes", "hrmap",
 * "submask" (field stop), "camimg" (uint16), "dark", "flat" (fakecam). */
int aob_sh_buffer(aob_sh *h, const char *which, void **dev_ptr, int64_t *nelem);
/* SutraWfsSH::comp_image(noise) (sutra_wfs_sh.cpp:623-643): fused field fill,
 * pruned 2-D DFT, |E|^2, binning, flux normalisation, photon/readout noise
 * and image scatter in one kernel.  If a centroider is attached with
 * aob_centro_attach_wfs, its slopes are computed in the same pass and kept
 * for the next aob_centro_get_cog on that centroider. */
int aob_sh_comp_image(aob_sh *h, int noise, void *stream);
/* SutraWfsSH::fill_binimage (sutra_wfs_sh.cpp:599-621): re-scatter bincube. */
int aob_sh_fill_binimage(aob_sh *h, void *stream);
/* Launch shape of the sensor kernel: sub-apertures per CTA batch (1..32;
 * 0 = heuristic).  Set by the project's autotuner; results are unchanged. */
int aob_sh_set_tuning(aob_sh *h, int subaps_per_cta);
/* set_bincube / set_binimg: overwrite from host. */
int aob_sh_set_bincube(aob_sh *h, const float *host, int64_t n);
int aob_sh_set_binimg(aob_sh *h, const float *host, int64_t n);
/* SutraWfs::slopes_geom(slopes, type) (sutra_wfs.cpp:199-251): geometric
 * slopes of the sensor's phase into dev_slopes (2 nvalid floats; NULL: the
 * sensor's own slopes buffer).  type 0: edge differences (phase_reduce), 1:
 * pupil-weighted finite differences over fluxPerSub (phase_derive), 2: the
 * tip/tilt projection matrix (phase_project).  Needs the phasemap (and for
 * type 2 ttprojmat) from load_arrays. */
int aob_sh_slopes_geom(aob_sh *h, int type, float *dev_slopes, void *stream);

/* ---- pyramid sensor ------------------------------------------------- *
 * Replaces SutraWfs_PyrHR (libsutra/src.cpp/sutra_wfs_pyr_pyrhr.cpp) as bound
 * by python_module/sutra/src/wfs_pyrhr.cpp:131-163.  npts modulation points,
 * nfft x nfft focal plane, ntot x ntot phase grid; binned image of
 * (nfft / nrebin)^2 pixels.                                               */
typedef struct aob_pyr aob_pyr;
/* Constructor arguments of SutraWfs_PyrHR (sutra_wfs_pyr_pyrhr.cpp:28-120);
 * npts is the reference's npup (number of modulation points). */
int aob_pyr_create(aob_pyr **out, int device, int nxsub, int nvalid, int npix, int nphase, int nrebin,
                   int nfft, int ntot, int npts, float pdiam, float nphot, float nphot4imat);
int aob_pyr_destroy(aob_pyr *h);
/* PYRWFS.load_arrays(halfxy, cx, cy, weights, sincar, submask, validsubsx,
 * validsubsy, phasemap, fluxPerSub, ttprojmat) (sutra_wfs_pyr_pyrhr.cpp:313-350):
 * halfxy = exp(i pyramid phase) as nfft^2 complex64 (float pairs), the
 * reference's layout; cx, cy, weights: npts modulation tilts / weights
 * (weights may be NULL = 1); sincar, submask: nfft^2; validsubsx / validsubsy:
 * 4 * nvalid; phasemap [nphase^2, nvalid] and ttprojmat [nphase^2, 2 nvalid]
 * (column-major, may be NULL) are kept for aob_pyr_slopes_geom. */
int aob_pyr_load_arrays(aob_pyr *h, const float *halfxy_c64, const float *cx, const float *cy,
                        const float *weights, const float *sincar, const float *submask,
                        const int32_t *validsubsx, const int32_t *validsubsy, const int32_t *phasemap,
                        const float *fluxPerSub, const float *ttprojmat);
/* set_pyr_modulation_points (sutra_wfs_pyr_pyrhr.cpp:695-720). */
int aob_pyr_set_modulation(aob_pyr *h, const float *cx, const float *cy, const float *weights, int npts);
int aob_pyr_set_pupil(aob_pyr *h, const float *pupil_host);
/* Photon (noise > -1) and readout (noise > 0) noise with the SH sensor's
 * Philox streams keyed by seed. */
int aob_pyr_set_noise(aob_pyr *h, float noise, int64_t seed);
int aob_pyr_set_lambda(aob_pyr *h, float lambda_um);
int aob_pyr_set_nphot(aob_pyr *h, float nphot);
int aob_pyr_set_frame(aob_pyr *h, uint64_t frame);
int aob_pyr_get_frame(aob_pyr *h, uint64_t *frame);
/* which: "phase", "pupil", "binimg", "hrimg", "validsubsx", "validsubsy",
 * "fluxPerSub", "submask", "phalfxy" (2 nfft^2 floats), "sincar", "phasemap",
 * "ttprojmat", "slopes" (geometric slopes), "pyrfocalplane" (nfft^2). */
int aob_pyr_buffer(aob_pyr *h, const char *which, void **dev_ptr, int64_t *nelem);
/* SutraWfs_PyrHR::comp_image(noise) (sutra_wfs_pyr_pyrhr.cpp:379-627). */
int aob_pyr_comp_image(aob_pyr *h, int noise, void *stream);
/* PYRWFS.set_submask (python_module/sutra/src/wfs_pyrhr.cpp:255-270,
 * sutra_wfs_pyr_pyrhr.cpp:361-377): the focal-plane field stop, nfft^2. */
int aob_pyr_set_submask(aob_pyr *h, const float *submask, int64_t n);
/* SutraWfs_PyrHR::set_phalfxy (sutra_wfs_pyr_pyrhr.cpp:731-744): the pyramid
 * mask exp(i phase), nfft^2 complex64 as float pairs (n = nfft^2). */
int aob_pyr_set_phalfxy(aob_pyr *h, const float *phalfxy_c64, int64_t n);
/* PYRWFS.set_pyrimg / set_binimg (wfs_pyrhr.cpp:190-205): the binned image. */
int aob_pyr_set_binimg(aob_pyr *h, const float *img, int64_t n);
/* PYRWFS.compute_pyrfocalplane (wfs_pyrhr.cpp:83-90): while enabled every
 * comp_image also forms the focal-plane image sum_p w_p |submask x focal
 * field_p|^2 (sutra_wfs_pyr_pyrhr.cpp:398-401) into "pyrfocalplane". */
int aob_pyr_set_compute_focalplane(aob_pyr *h, int enable);
/* SutraWfs::slopes_geom for the pyramid sensor (see aob_sh_slopes_geom);
 * dev_slopes NULL: the sensor's "slopes" buffer. */
int aob_pyr_slopes_geom(aob_pyr *h, int type, float *dev_slopes, void *stream);

/* ---- centroiders ------------------------------------------------------ *
 * Replaces SutraCentroiderCog / Tcog / Wcog (libsutra/src.cpp/
 * sutra_centroider_{cog,tcog,wcog}.cpp, kernels sutra_centroider_*.cu) as
 * bound by python_module/sutra/src/centroider*.cpp.                      */
typedef struct aob_centro aob_centro;
#define AOB_CENTRO_COG 0
#define AOB_CENTRO_TCOG 1
#define AOB_CENTRO_WCOG 2
#define AOB_CENTRO_PYR 3
/* SutraCentroiderMaskedPix (sutra_centroider_maskedPix.cpp, kernel
 * sutra_centroider_maskedPix.cu:26-56): one slope per valid pixel,
 * s[i] = pix[i] / sum(pix) * n - ref[i]; nvalid is the number of pixels (4 *
 * the pyramid's nvalid) and the reference slopes start at 1. */
#define AOB_CENTRO_MASKEDPIX 4
/* SutraCentroiderBpcog (sutra_centroider_bpcog.cu:24-80): CoG over the pixels
 * above the value of rank nmax (aob_centro_set_nmax), thresholded pixels
 * written back into the image. */
#define AOB_CENTRO_BPCOG 5
#define AOB_SLOPES_UNTIED 0
#define AOB_SLOPES_INTERLEAVED 1

/* SutraRtc::add_centroider (libsutra/src.cpp/sutra_rtc.cpp:64-111). */
int aob_centro_create(aob_centro **out, int device, int type, int nvalid, float offset,
                      float scale);
int aob_centro_destroy(aob_centro *c);
/* Bind to a SH sensor: the centroider reads its binimg (SutraCentroider
 * ctor, sutra_centroider.cpp:42-46) and its slopes are fused into
 * aob_sh_comp_image. */
int aob_centro_attach_wfs(aob_centro *c, aob_sh *h);
int aob_centro_set_npix(aob_centro *c, int npix);
int aob_centro_set_scale(aob_centro *c, float scale);
int aob_centro_set_offset(aob_centro *c, float offset);
int aob_centro_set_threshold(aob_centro *c, float threshold);
int aob_centro_set_slope_order(aob_centro *c, int order);
/* Pyramid centroider (type AOB_CENTRO_PYR, SutraCentroiderPyr::get_pyr,
 * libsutra/src.cpp/sutra_centroider_pyr.cpp:101-130): reads the binned image
 * of the attached pyramid sensor (a masked-pixel centroider may be attached
 * to one too); its valid positions are 4 * nvalid pixels
 * (quadrant k of sub-aperture i at entry i + k nvalid).  method (set_pyr_method,
 * python_module/sutra/src/centroider_pyr.cpp:35-64), decoded as the reference's
 * Method_CoG(uint8_t) does (libsutra/include/sutra_centroider_pyr.hpp:27-34):
 * 0 sinus global, 1 nosinus global (the default), 2 sinus local (per
 * sub-aperture flux), 3 nosinus local.  thresh: flux below which the slopes
 * are 0 (reference default 1e-4). */
int aob_centro_attach_pyr(aob_centro *c, aob_pyr *p);
/* set_nmax (python_module/sutra/src/centroider_bpcog.cpp): rank of the
 * threshold pixel of a bpcog centroider, 0 <= nmax < 1024. */
int aob_centro_set_nmax(aob_centro *c, int nmax);
int aob_centro_set_pyr_method(aob_centro *c, int method);
int aob_centro_set_pyr_thresh(aob_centro *c, float thresh);
/* load_validpos (sutra_centroider.cpp:287-298); n = nvalid (4 * nvalid for a
 * pyramid centroider). */
int aob_centro_load_validpos(aob_centro *c, const int32_t *validx, const int32_t *validy, int n);
/* set_centroids_ref (sutra_centroider.cpp:300-304). */
int aob_centro_set_centroids_ref(aob_centro *c, const float *ref);
/* wCoG weights: n == npix*npix (one map for all sub-apertures) or
 * npix*npix*nvalid (sutra_centroider_wcog.cpp:47-75). */
int aob_centro_load_weights(aob_centro *c, const float *weights, int64_t n);
/* load_img / set_dark / set_flat / calibrate_img (sutra_centroider.cpp:
 * 233-285,120-140,200-230): image of m x n pixels from host. */
int aob_centro_load_img(aob_centro *c, const float *img, int m, int n);
int aob_centro_set_dark(aob_centro *c, const float *dark, int n);
int aob_centro_set_flat(aob_centro *c, const float *flat, int n);
int aob_centro_calibrate_img(aob_centro *c, void *stream);
/* The camera path (Rtc_UFF: uint16 input, SutraCentroider<uint16_t, float>,
 * sutra_centroider.cpp:246-285): load_img of an m x n uint16 frame from host
 * (on_device 0; the call waits for the copy) or device memory.  calibrate_img
 * then gives float (raw[lut] - dark) * flat (calib_krnl,
 * libsutra/src.cu/sutra_centroider.cu:108-115); "img_raw" returns the last
 * loaded frame in its type. */
int aob_centro_load_img_u16(aob_centro *c, const uint16_t *img, int m, int n, int on_device, void *stream);
/* set_lutPix (sutra_centroider.cpp:163-172): raw pixel read for each image
 * pixel (identity until set), n = m * n entries, each < n. */
int aob_centro_set_lut_pix(aob_centro *c, const int32_t *lut, int n);
/* calibrate_img_validPix (sutra_centroider.cpp:194-223): the calibration on the
 * valid pixels only (SH: the npix x npix window of each valid sub-aperture;
 * pyramid and masked-pixel: each listed pixel), the rest of the image zero. */
int aob_centro_calibrate_img_validpix(aob_centro *c, void *stream);
/* get_cog (sutra_centroider_cog.cpp:51-98): slopes into dev_slopes (2*nvalid
 * floats, device) and intensities into the centroider's buffer. */
int aob_centro_get_cog(aob_centro *c, float *dev_slopes, void *stream);
int aob_centro_buffer(aob_centro *c, const char *which, void **dev_ptr, int64_t *nelem);
int aob_centro_get_params(aob_centro *c, int *type, int *nvalid, int *npix, float *offset,
                          float *scale, float *threshold);

/* ---- least-squares controller ------------------------------------------ *
 * Replaces SutraControllerLs + SutraController (libsutra/src.cpp/
 * sutra_controller_ls.cpp, sutra_controller.cpp) as bound by
 * python_module/sutra/src/controller_ls.cpp:69-245 and controller.cpp.    */
typedef struct aob_ls aob_ls;
#define AOB_PREC_F32 0
#define AOB_PREC_BF16 1
#define AOB_PREC_FP8 2

int aob_ls_create(aob_ls **out, int device, int nslope, int nactu, float delay);
int aob_ls_destroy(aob_ls *c);
/* set_cmat (sutra_controller_ls.cpp:152-157): column-major [nactu, nslope]. */
int aob_ls_set_cmat(aob_ls *c, const float *cmat);
int aob_ls_set_imat(aob_ls *c, const float *imat);
/* set_modal_gains (sutra_controller_ls.cpp:166-171). */
int aob_ls_set_modal_gains(aob_ls *c, const float *gains);
int aob_ls_set_gain(aob_ls *c, float gain);
int aob_ls_set_delay(aob_ls *c, float delay);
int aob_ls_set_open_loop(aob_ls *c, int open_loop, int reset);
int aob_ls_set_com_range(aob_ls *c, float volt_min, float volt_max);
int aob_ls_set_com(aob_ls *c, const float *com, int n);
int aob_ls_set_centroids(aob_ls *c, const float *s, int n);
/* Precision of the command-matrix MVM: F32 (reference), BF16, or FP8 E4M3
 * with one float32 scale per actuator row; accumulation is always float32. */
int aob_ls_set_precision(aob_ls *c, int prec);
/* MVM kernel choice: kind 0 = auto, 1 = bulk-copy (TMA) staging of the
 * CTA's rows in shared memory, 2 = register streaming; nblocks = grid size
 * (0 = one CTA per SM).  Set by the autotuner; results are unchanged. */
int aob_ls_set_tuning(aob_ls *c, int kind, int nblocks);
/* Error word of the MVM kernels (bit 0: a bounded wait expired); reset = clear it. */
int aob_ls_status(aob_ls *c, uint32_t *status, int reset);
/* comp_com (sutra_controller_ls.cpp:251-285): err = -cmat.s,
 * com += gain * err * modal_gains, one kernel. */
int aob_ls_comp_com(aob_ls *c, void *stream);
/* clip_commands (sutra_controller.cpp:221-229). */
int aob_ls_clip(aob_ls *c, void *stream);
/* comp_voltage (sutra_controller.cpp:245-263): latency interpolation,
 * command delay ring, perturbation voltages, clip. */
int aob_ls_comp_voltage(aob_ls *c, void *stream);
/* Perturbation voltages (sutra_controller.cpp:98-195): perturb is
 * [N, nactu] column-major. */
int aob_ls_add_perturb(aob_ls *c, const char *name, const float *perturb, int n);
int aob_ls_remove_perturb(aob_ls *c, const char *name);
int aob_ls_enable_perturb(aob_ls *c, const char *name, int enable);
int aob_ls_reset_perturb(aob_ls *c);
/* add_perturb (sutra_controller.cpp:266-285): com_clipped += the current row
 * of every enabled perturbation buffer, whose counter then advances (the step
 * comp_voltage runs before its clip). */
int aob_ls_apply_perturb(aob_ls *c, void *stream);
/* One SVD-style eigen decomposition of imat^T imat in float64 on the GPU
 * (svdec_imat, sutra_controller_ls.cpp:116-150) and the filtered
 * pseudo-inverse (build_cmat, :174-217). */
int aob_ls_svdec_imat(aob_ls *c);
int aob_ls_build_cmat(aob_ls *c, int nfilt);
/* which: "centroids", "com", "com_clipped", "voltage", "err", "cmat",
 * "imat", "eigenvals", "gain", "com0", "com1". */
int aob_ls_buffer(aob_ls *c, const char *which, void **dev_ptr, int64_t *nelem);
int aob_ls_get_params(aob_ls *c, int *nslope, int *nactu, float *delay, float *gain,
                      int *open_loop, float *volt_min, float *volt_max, int *prec);

/* ---- generic controller ------------------------------------------------- *
 * Replaces SutraControllerGeneric (libsutra/src.cpp/sutra_controller_generic.cpp,
 * bound by python_module/sutra/src/controller_generic.cpp).  It is an aob_ls
 * handle of kind AOB_CTRL_GENERIC: every aob_ls_* call applies (cmat, gain,
 * modal gains, delay, perturbation, clip, comp_voltage, buffers), and comp_com
 * runs its command law (comp_com, sutra_controller_generic.cpp:219-328):
 *   AOB_LAW_INTEGRATOR        com = berta com - gain cmat s
 *   AOB_LAW_MODAL_INTEGRATOR  b = -(cmat s) * modal gains; com = gain matE b + berta com
 *   AOB_LAW_2MATRICES         b = -(cmat s) * modal gains; com = (matE com1) * decay + b
 * with berta = the leaky factor, or with pseudo-open-loop control (polc: s
 * replaced by s - imat com_clipped) (1 - gain) * leaky; com1 is the previous
 * command.  The gain starts at 0, the leaky factor at 1.  No state vector
 * (nstates = 0).  The fused RTC kernel and the batch take LS controllers only. */
#define AOB_CTRL_LS 0
#define AOB_CTRL_GENERIC 1
#define AOB_LAW_INTEGRATOR 1
#define AOB_LAW_MODAL_INTEGRATOR 2
#define AOB_LAW_2MATRICES 3
int aob_generic_create(aob_ls **out, int device, int nslope, int nactu, float delay);
/* kind (AOB_CTRL_*), command law, leaky factor, polc flag. */
int aob_ls_get_kind(aob_ls *c, int *kind, int *law, float *leaky, int *polc);
/* set_commandlaw / set_leaky_factor / set_polc (controller_generic.cpp). */
int aob_ls_set_commandlaw(aob_ls *c, int law);
int aob_ls_set_leaky_factor(aob_ls *c, float leaky);
int aob_ls_set_polc(aob_ls *c, int polc);
/* set_decayFactor (nactu) and set_matE (nactu x nactu, column-major). */
int aob_ls_set_decay_factor(aob_ls *c, const float *decay);
int aob_ls_set_matE(aob_ls *c, const float *matE);


/* ---- learned reconstructor (MLP) ---------------------------------------- *
 * No counterpart in the reference.  A 3-layer MLP slopes -> DM commands
 * (nin -> nh1 -> nh2 -> nout, GELU on the hidden layers), BF16 weights and
 * activations with FP32 accumulation, trained on the GPU (tensor-core GEMMs,
 * Adam).  The network works on x = slopes * in_scale and predicts
 * commands / out_scale.  Weights are row-major [out][in] float32 on the host. */
typedef struct aob_mlp aob_mlp;
int aob_mlp_create(aob_mlp **out, int device, int nin, int nh1, int nh2, int nout);
int aob_mlp_destroy(aob_mlp *m);
/* layer 0, 1, 2: W [rows][cols] and b [rows]; resets the optimiser state. */
int aob_mlp_set_params(aob_mlp *m, int layer, const float *w, const float *b);
int aob_mlp_get_params(aob_mlp *m, int layer, float *w, float *b);
int aob_mlp_set_scales(aob_mlp *m, float in_scale, float out_scale);
/* Batched forward: dev_x [batch][nin] slopes -> dev_y [batch][nout] commands
 * (dev_y may be NULL: the outputs stay in the network's buffer "y"). */
int aob_mlp_forward(aob_mlp *m, const float *dev_x, int batch, float *dev_y, void *stream);
/* Gradients of the mean-squared error against dev_target [batch][nout]
 * (commands) after aob_mlp_forward on the same batch; dev_loss (may be NULL)
 * receives the loss on the scaled outputs.  Buffers "dW1".."dW3", "db1".."db3". */
int aob_mlp_backward(aob_mlp *m, const float *dev_target, int batch, float *dev_loss, void *stream);
/* forward + backward + one Adam step with learning rate lr. */
int aob_mlp_train_step(aob_mlp *m, const float *dev_x, const float *dev_target, int batch, float lr,
                       float *dev_loss, void *stream);
/* Batch-1 inference (GEMV kernels): dev_x [nin] -> dev_y [nout]. */
int aob_mlp_infer(aob_mlp *m, const float *dev_x, float *dev_y, void *stream);
/* Controller step with the learned reconstructor: commands c = MLP(centroids
 * of ls); if ||c|| <= threshold, err = -c and the integrator of ls is applied,
 * otherwise ls's own MVM runs (LS fallback, counted).  Then call
 * aob_ls_comp_voltage as usual. */
int aob_mlp_comp_com(aob_mlp *m, aob_ls *ls, float threshold, void *stream);
/* Control-step path: 0 = one cooperative kernel (all layers, the threshold
 * test and the LS fallback in one launch; weights streamed into shared memory
 * at entry) whenever it fits, 1 = the multi-kernel path (GEMV per layer,
 * select, LS MVM).  The commands are the same bit for bit. */
int aob_mlp_set_mode(aob_mlp *m, int mode);
/* Training GEMMs: 0 = mma.sync kernel (128 x 128 x 32 tiles), 1 = tcgen05
 * kernel (TMA tensor loads, 128 x 128 FP32 accumulator in TMEM; the default). */
int aob_mlp_set_gemm(aob_mlp *m, int kind);
/* Error word of the tcgen05 GEMM's bounded waits (bit 3: a wait expired). */
int aob_mlp_gemm_status(aob_mlp *m, uint32_t *status, int reset);
/* Number of LS fallbacks so far (reset != 0: set it back to 0). */
int aob_mlp_fallbacks(aob_mlp *m, uint32_t *count, int reset);
/* which: "W1".."W3", "b1".."b3" (FP32 masters, padded), "dW1".."dW3", "db1".."db3", "y". */
int aob_mlp_buffer(aob_mlp *m, const char *which, void **dev_ptr, int64_t *nelem);
/* Padded sizes {nin, nh1, nh2, nout} (multiples of 8). */
int aob_mlp_get_dims(aob_mlp *m, int *padded4);

/* ---- batched 2-D FFT ---------------------------------------------------- *
 * In-place complex64 n x n transforms of `batch` contiguous images, n a power
 * of two in [8, 2048]; cuFFT sign convention (forward = exp(-i...)),
 * unnormalised.  Replaces the CarmaFFT calls of the target and pyramid paths
 * (libcarma/src.cpp/carma_fft.cpp:165-179). */
int aob_fft2d_c64(void *dev_data, int n, int batch, int inverse, int device, void *stream);

/* ---- turbulent layers ----------------------------------------------------- *
 * Replaces SutraAtmos / SutraTurbuScreen (libsutra/src.cpp/sutra_atmos.cpp,
 * sutra_tscreen.cpp) as bound by python_module/sutra/src/atmos.cpp. */
typedef struct aob_atmos aob_atmos;
int aob_atmos_create(aob_atmos **out, int device);
int aob_atmos_destroy(aob_atmos *a);
/* add_screen + init_screen (sutra_atmos.cpp:52-81): A is dim x nstencil and B
 * dim x dim, column-major; istx/isty index the flattened screen; r0 in pixels. */
int aob_atmos_add_screen(aob_atmos *a, int dim, int nstencil, float r0_pix, float altitude, float deltax,
                         float deltay, const float *A, const float *B, const uint32_t *istx,
                         const uint32_t *isty, int64_t seed, int *index);
/* refresh_screen (sutra_tscreen.cpp:113-127): zero, then 2*dim extrusions. */
int aob_atmos_refresh_screen(aob_atmos *a, int idx, void *stream);
/* move_atmos (sutra_atmos.cpp:82-100). */
int aob_atmos_move(aob_atmos *a, void *stream);
/* Current screen of layer idx (device pointer changes after each extrusion). */
int aob_atmos_screen(aob_atmos *a, int idx, void **dev_screen, int *dim, float *accumx, float *accumy);
int aob_atmos_nscreens(aob_atmos *a, int *n);
/* Float64 factorisation of the extrusion operators on the GPU (iterkolmo.AB,
 * shesha/shesha/util/iterkolmo.py:225-251) from the host covariances zz
 * (nst x nst), xz (n x nst), xx (n x n), column-major; outputs A (n x nst) and
 * B (n x n) column-major float32. */
int aob_kolmo_factor_ab(int device, int n, int nst, const double *zz, const double *xz, const double *xx,
                        float *A, float *B);

/* Allocation-free extrusion: no counterpart in the reference.  For callers that
 * may not allocate device memory while they run -- a real-time controller with
 * all memory reserved at start-up (cudaMalloc / cudaFree synchronise the device
 * and take an unbounded time) or a plugin inside a host that owns the device
 * memory.  Extrudes the caller's n x n screen (x fastest, updated in place) by
 * one column (direction +-1) or row (+-2), exactly like one step of
 * aob_atmos_move: A is n x nstencil and B n x n stored ROW-major (row i
 * contiguous, the transpose of the column-major arrays aob_atmos_add_screen
 * takes), dev_stencil holds nstencil indexes < n*n, amplitude is
 * r0_pix^(-5/6) * 0.5 / (2 pi), and (seed, counter, layer_index) select the
 * noise exactly as the layer's extrusion counter and index do there.
 * Limit: n <= AOB_NOALLOC_EXTRUDE_MAX_N; larger n is rejected with AOB_ERR.
 * The scratch is one fixed device array (about 1 MB, held by every GPU that
 * loads the library until exit) shared by all calls: calls that overlap on the
 * GPU (other streams, other host threads) race on it -- order them.  The first
 * call on a device looks the array's address up (cudaGetSymbolAddress); make
 * that first call before any stream capture.  The address is kept for the
 * life of the process: after cudaDeviceReset (or another teardown of the
 * device's primary context) do not call this entry point on that device
 * again.  The stencil indexes are not checked on the device (a caller
 * precondition, as stated above).  The caller's current device is left as it
 * was. */
#define AOB_NOALLOC_EXTRUDE_MAX_N 512
int aob_extrude_noalloc(float *dev_screen, int n, int nstencil, const float *dev_A_rows,
                        const float *dev_B_rows, const uint32_t *dev_stencil, int direction, float amplitude,
                        int64_t seed, uint32_t counter, int layer_index, int device, void *stream);

/* ---- deformable mirror ---------------------------------------------------- *
 * Replaces SutraDm (pzt) as loaded by pzt_loadarrays
 * (libsutra/src.cpp/sutra_dm.cpp) and shaped by comp_shape (sutra_dm.cu:43-133). */
typedef struct aob_dm aob_dm;
/* influ: influsize x influsize x nact (Fortran order); i1/j1: lower-left pixel of
 * each influence patch in the dim x dim DM screen. */
int aob_dm_create(aob_dm **out, int device, int dim, int nact, int influsize, const float *influ,
                  const int32_t *i1, const int32_t *j1);
int aob_dm_destroy(aob_dm *d);
/* dev_com: nact commands on the device (NULL = the DM's own command buffer). */
int aob_dm_comp_shape(aob_dm *d, const float *dev_com, void *stream);
/* which: "shape", "com". */
int aob_dm_buffer(aob_dm *d, const char *which, void **dev_ptr, int64_t *nelem);

/* ---- interaction matrix ------------------------------------------------------ *
 * SutraRtc::do_imat (libsutra/src.cpp/sutra_rtc.cpp:150-292), every actuator of
 * the DM poked in one batch: the push (+push) and pull (-push) DM shapes of a
 * chunk of actuators (chunk 0 = all), their bilinear raytrace onto the sensor's
 * npup x npup phase grid at offset (xoff, yoff) in the DM screen, the sensor
 * images with the attached CoG-family centroider over all pokes in one launch
 * (noise-free, with the sensor's nphot4imat photons when it is > 0 as
 * SutraRtc::comp_images_imat does, else its current photon count), and the columns
 * (s_push - s_pull) / (2 push) into dev_imat, nslope x nact column-major on the
 * device.  Equal bit for bit to poking one actuator after the other with
 * aob_dm_comp_shape, aob_raytrace, aob_sh_comp_image and aob_centro_get_cog
 * (at the same photon count).
 * Needs about 2 chunk (dim^2 + npup^2) floats of scratch; waits for the stream. */
int aob_imat_build(aob_sh *w, aob_centro *c, aob_dm *dm, float xoff, float yoff, float push, int chunk,
                   float *dev_imat, void *stream);

/* ---- raytracing ------------------------------------------------------------ *
 * SutraSource::raytrace (libsutra/src.cpp/sutra_source.cpp:222-320) with the
 * bilinear generic_raytrace (sutra_target.cu:25-70): out (nx x ny) = (reset ? 0 :
 * out) + sum over nsrc screens of screen_k sampled at (x + xoff_k, y + yoff_k).
 * nsrc <= 8. */
int aob_raytrace(float *dev_out, int nx, int ny, int nsrc, const float *const *dev_screens, const int *dims,
                 const float *xoff, const float *yoff, int reset, void *stream);

/* ---- science target -------------------------------------------------------- *
 * SutraSource::comp_image / comp_strehl (sutra_source.cpp:397-515): short- and
 * long-exposure PSF normalised so that the peak is the Strehl ratio; the peak
 * read directly (aob_target_strehl) or by the reference's sinc fit
 * (aob_target_strehl_fit). */
typedef struct aob_target aob_target;
int aob_target_create(aob_target **out, int device, int npup, int nfft, const float *pupil, float lambda_um);
int aob_target_destroy(aob_target *t);
/* dev_phase: npup x npup phase in micron (NULL = the target's own buffer). */
int aob_target_comp_image(aob_target *t, const float *dev_phase, int comp_le, void *stream);
int aob_target_strehl(aob_target *t, float *se, float *le, void *stream);
/* comp_strehl(do_fit = true) (sutra_source.cpp:491-515, fitmax2x1dSinc
 * :451-488): the peak of each image estimated by a sinc (Shannon) interpolation
 * at the sub-pixel maximum that parabolas through the 3-pixel cross around the
 * brightest pixel give, over its 7 x 7 periodic window; the long exposure is
 * divided by the number of images summed.  Waits for the stream. */
int aob_target_strehl_fit(aob_target *t, float *se, float *le, void *stream);
int aob_target_reset_le(aob_target *t, void *stream);
/* which: "phase", "image_se", "image_le", "amplipup". */
int aob_target_buffer(aob_target *t, const char *which, void **dev_ptr, int64_t *nelem);

/* ---- one closed-loop RTC iteration ------------------------------------ *
 * The per-iteration RTC sequence that CompassSupervisor.next() drives
 * through separate calls (shesha/shesha/supervisor/compassSupervisor.py:
 * 175-289: compute_wfs_image -> do_centroids -> do_control -> apply_control
 * with comp_voltage), bound into one object so that it runs as three kernels
 * (SH image + fused centroids, MVM + integrator, voltage) with the slopes
 * written straight into the controller's input. */
typedef struct aob_loop aob_loop;
int aob_loop_create(aob_loop **out, aob_sh *wfs, aob_centro *centro, aob_ls *ls);
int aob_loop_destroy(aob_loop *l);
/* One iteration.  host_phase (npup*npup floats, may be NULL = use the
 * sensor's current device phase) is copied in first; host_voltage (nactu
 * floats, may be NULL) receives the voltages, and the call then waits for
 * the stream.  noise != 0 adds photon/readout noise. */
int aob_loop_step(aob_loop *l, const float *host_phase, float *host_voltage, int noise, void *stream);
/* The same step without the final wait: the phase copy, the kernels and the
 * voltages' way back to host_voltage are enqueued on the stream and the call
 * returns.  The voltages are valid once the stream has reached this point (an
 * event or a synchronisation); host_phase must stay unchanged until then.  With
 * pinned host buffers nothing in the call blocks the host (pageable buffers make
 * the copies synchronous).  For callers that step many iterations and read the
 * results later, as the reference's supervisor loop does between frames. */
int aob_loop_step_async(aob_loop *l, const float *host_phase, float *host_voltage, int noise, void *stream);
/* nsteps iterations streamed from the host: no single counterpart in the
 * reference, whose supervisor calls set_phase, comp_image, do_centroids,
 * do_control and comp_voltage once per frame (CompassSupervisor.next,
 * shesha/shesha/supervisor/compassSupervisor.py:175); this is
 * nsteps of those frames in one call.  Step k takes host_phases[k % nphases]
 * (nphases phases of npup*npup floats back to back) and writes its voltages to
 * host_voltages + k*nactu (may be NULL).  The kernels and their order are those
 * of nsteps aob_loop_step calls, so the voltages are the same bit for bit; the
 * phase of step k+1 is copied to the device on a stream of the loop's own while
 * step k computes.  Host buffers should be pinned: pageable ones make the copies
 * synchronous and remove the overlap.  wait != 0 waits for the stream at the end;
 * otherwise host_phases must stay unchanged and host_voltages unread until the
 * stream reaches that point. */
int aob_loop_run(aob_loop *l, const float *host_phases, int nphases, int nsteps, float *host_voltages, int noise,
                 void *stream, int wait);
/* One iteration with the learned reconstructor m in place of the LS matrix (no
 * counterpart in the reference, whose reconstructors are linear): the sensor
 * image with fused centroids into the controller, aob_mlp_comp_com's control
 * step (the network, the threshold test, then the integrator or the LS
 * fallback on the controller's own matrix), the voltages.  Host buffers as in
 * aob_loop_step.  With an FP32 LS matrix and a configuration that fits, one
 * cooperative kernel does all of it (rtc_mlp_kernel), else separate launches;
 * the results are the same bit for bit.  The network's sizes must be the
 * controller's (nin = nslope, nout = nactu). */
int aob_loop_step_mlp(aob_loop *l, aob_mlp *m, float threshold, const float *host_phase, float *host_voltage,
                      int noise, void *stream);
/* The same without the final wait (as aob_loop_step_async). */
int aob_loop_step_mlp_async(aob_loop *l, aob_mlp *m, float threshold, const float *host_phase,
                            float *host_voltage, int noise, void *stream);
/* Persistent mode (no counterpart in the reference): the fused kernel stays
 * resident -- its command-matrix rows, sensor tables and the integrator state
 * in shared memory -- and runs one RTC step per doorbell.  persist_start
 * launches it (noise: the setting every step uses; host_voltage: pinned,
 * mapped host memory the kernel writes the voltages into at every step, or
 * NULL; door_polls: limit of one wait for a doorbell, 0 = about two seconds,
 * after which the kernel leaves and sets bit 4 (16) of aob_ls_status).
 * persist_step enqueues one step on stream: the host phase copy (if given), a
 * stream write of the step's doorbell, a stream wait until the kernel reports
 * it done, and the voltages into host_voltage (copied unless it is the
 * buffer given to persist_start); wait = 1 also synchronises.  Results equal
 * aob_loop_step's bit for bit.  persist_stop lets the kernel leave after the
 * steps already rung.  While the kernel runs, the sensor, centroider and
 * controller must not be changed or stepped otherwise; the controller must
 * have no delay, and nothing may synchronise the whole device (it would wait
 * for the resident kernel until its doorbell wait runs out): synchronise
 * streams.  Needs the driver's stream memory operations. */
int aob_loop_persist_start(aob_loop *l, int noise, float *host_voltage, uint32_t door_polls);
int aob_loop_persist_step(aob_loop *l, const float *host_phase, float *host_voltage, int noise, void *stream,
                          int wait);
int aob_loop_persist_stop(aob_loop *l);
/* While the kernel is resident it holds every SM's registers, so no other
 * kernel runs beside it: persist_flush has the resident kernel itself write
 * bytes of zeros over dev_buf (16-byte aligned, a multiple of 16 bytes), e.g.
 * to flush L2 between timed steps of a benchmark.  Enqueued on stream like a
 * step; it does not count as an RTC step (no noise frame). */
int aob_loop_persist_flush(aob_loop *l, void *dev_buf, size_t bytes, void *stream);
/* The resident kernel's own account of its RTC steps since persist_start:
 * the number of steps rung and the sum of their busy times in nanoseconds
 * (GPU global timer, from the doorbell seen by CTA 0 to the step's done). */
int aob_loop_persist_stats(aob_loop *l, uint64_t *steps, uint64_t *busy_ns);

/* Device time of one step (ms, CUDA events on a private stream; device
 * phase, no host copies): warmup untimed steps, then the mean over iters
 * steps.  Used by the autotuner; the loop state advances. */
int aob_loop_time(aob_loop *l, int noise, int warmup, int iters, float *ms_per_step);
/* Replay the device part of a step from a CUDA graph (enable != 0).  Applies
 * to the three-kernel step; the fused single-kernel step is always launched
 * directly (a one-node graph only adds launch latency). */
int aob_loop_use_graph(aob_loop *l, int enable);
/* Kernels launched by the device part of the last step. */
int aob_loop_kernels_per_step(aob_loop *l, int *n);
/* mode 0 = fused single cooperative kernel when the configuration fits
 * (otherwise three kernels), 1 = always three kernels, 2 = fused only (error
 * if it does not fit); fused_batch = at most this many sub-apertures per CTA
 * and round in the fused kernel (0 = a CTA's whole share in one round). */
int aob_loop_set_mode(aob_loop *l, int mode, int fused_batch);
/* Voltage output of aob_loop_step: mode 1 (default) = when host_voltage is
 * pinned, mapped host memory and the fused kernel runs, its epilogue writes
 * the voltages there directly (no copy-engine transfer after the kernel);
 * mode 0 = always a device-to-host copy.  Results are identical.  No
 * counterpart in the reference, whose controller keeps its voltages in device
 * memory (d_voltage) for the DMs. */
int aob_loop_set_host_io(aob_loop *l, int mode);

/* Test of the bounded grid-barrier wait (no counterpart in the reference):
 * one noise-free fused step in which CTA 0 never arrives at the barrier, so
 * the other CTAs' waits (at most `polls` polls each) expire.  Every CTA then
 * skips the MVM and returns, the kernel sets bit 1 (2, grid wait expired) of
 * the controller's status word (aob_ls_status), the arrival counter is
 * re-armed on the stream and the call waits for the stream.  The commands and
 * voltages are left as they were; later steps run normally.  Needs a
 * configuration that runs the fused kernel and a controller with delay 0. */
int aob_loop_test_wait_expiry(aob_loop *l, uint32_t polls, void *stream);

/* ---- batched Monte Carlo: many loops, one persistent launch per step --- *
 * No counterpart in the reference, where each simulation is its own process
 * stepping its own objects (CompassSupervisor.next, shesha/shesha/supervisor/
 * compassSupervisor.py:175-289).  A batch holds any number of SH loops of
 * uneven size (Nfft 16 or 32, any pixels, any MVM precision; controller delay
 * 0, no perturbation) and advances all of them with ONE kernel launch, replayed
 * from a CUDA graph: a queue of sensor items (runs of sub-apertures) and MVM
 * items (blocks of command-matrix rows) taken by persistent CTAs, with the MVM
 * items of an instance waiting (bounded) for its sensor items.  Results are
 * bit-identical to stepping each loop with aob_loop_step.  Parameters are
 * snapshot when the batch is (re)built: automatically on the first step and
 * when a loop's graph-relevant parameters change; aob_batch_refresh forces it.
 * Status bits of expired waits: 1 row copy, 4 sensor-item dependency. */
typedef struct aob_batch aob_batch;
int aob_batch_create(aob_batch **out, int device);
int aob_batch_destroy(aob_batch *b);
/* The loop must outlive the batch. */
int aob_batch_add(aob_batch *b, aob_loop *loop);
/* Tile shapes (the autotuner's choice): sub-apertures per sensor item (0 =
 * 32, at most 1024), threads per sensor team (0 = 32; 32, 64, 128 or 256: an
 * item's sub-apertures are shared by the CTA's teams, each runs its share as
 * one batch), command-matrix KB per MVM item (0 = 48, at most 200), lag in
 * instances between an instance's sensor and MVM items, CTAs per SM (0 = 2,
 * at most 4), instance order (0 = largest first, 1 = as added). */
int aob_batch_set_tuning(aob_batch *b, int subaps_per_item, int team_threads, int mvm_kb, int lag, int ctas_per_sm,
                         int order);
int aob_batch_use_graph(aob_batch *b, int enable);
/* Test of the bounded dependency wait: one step (direct launch) in which every
 * MVM item waits for one sensor item more than its instance has, so each such
 * wait expires after `polls` polls, the item skips its rows and the status
 * word gets bit 2 (4).  The queue re-arms itself as after any step; the status
 * word is cleared by the next rebuild (aob_batch_refresh).  Waits for the stream. */
int aob_batch_test_wait_expiry(aob_batch *b, uint32_t polls, int noise, void *stream);
int aob_batch_refresh(aob_batch *b);
/* One step of every loop with phases from each sensor's own device buffer. */
int aob_batch_step(aob_batch *b, int noise, void *stream);
/* One step with host I/O: host_phases (all sensors' npup*npup phases
 * concatenated in insertion order; NULL = device phases) are copied in,
 * host_volts (all nactu voltages concatenated; may be NULL) receive the
 * voltages, and the call waits for the stream. */
int aob_batch_step_host(aob_batch *b, const float *host_phases, float *host_volts, int noise, void *stream);
/* info[0..n): instances, queue items, CTAs, shared bytes per CTA, rows per
 * MVM item (max), algorithmic HBM bytes per step, phase floats, voltage floats. */
int aob_batch_info(aob_batch *b, int64_t *info, int n);
/* Offsets of each instance in the concatenated phase / voltage arrays. */
int aob_batch_offsets(aob_batch *b, int64_t *phase_off, int64_t *volt_off);
int aob_batch_status(aob_batch *b, uint32_t *status);
/* Device time of one step (ms, CUDA events on a private stream): warmup
 * untimed steps, then the mean over iters steps.  Used by the autotuner. */
int aob_batch_time(aob_batch *b, int noise, int warmup, int iters, float *ms_per_step);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif
#ifdef __cplusplus
}
#endif
#endif /* AOB200_H */
