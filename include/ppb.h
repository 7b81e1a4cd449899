/*
 * ppb.h — C ABI of libppb, a B200 (sm_100a) implementation of PeakPatch.jl's
 * per-tile halo-finding path.
 *
 * Every entry point returns an int32 status (PPB_OK or a negative PPB_ERR_*
 * code); no C++ exception crosses this boundary.  On failure the context
 * keeps a message retrievable with ppb_last_error().
 *
 * Conventions shared with the reference (PeakPatch.jl):
 *  - 3-D fields are n1 x n2 x n3 Float32 arrays in column-major order
 *    (i fastest), exactly as Julia stores Array{Float32,3}.
 *  - Peak indices i, j, k and the flat index ipp are 1-based
 *    (ipp = i + (j-1) n1 + (k-1) n1 n2), as in PeakFind.PeakCandidate.
 *  - "No collapse" is RTHL = -1 and zvir_half = -1 (RadialShell.no_collapse).
 *  - Pointers may be host or device memory: the library asks the CUDA driver
 *    which one it was given and copies host data in and out itself.  The
 *    caller keeps ownership of every buffer it passes.
 *
 * Reference interfaces each entry point replaces are cited per function
 * (paths inside the PeakPatch.jl repository).
 */
#ifndef PPB_H
#define PPB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PPB_ABI_VERSION 5

enum {
  PPB_OK = 0,
  PPB_ERR_INVALID = -1,      /* bad argument (null pointer, size out of range, ...) */
  PPB_ERR_CUDA = -2,         /* a CUDA runtime / cuFFT call failed */
  PPB_ERR_NOMEM = -3,        /* device allocation failed */
  PPB_ERR_ADMISSION = -4,    /* request larger than the context's HBM budget */
  PPB_ERR_TIMEOUT = -5,      /* a bounded wait ran out */
  PPB_ERR_UNSUPPORTED = -6,  /* option not implemented on this path */
  PPB_ERR_CAPACITY = -7,     /* caller buffer too small; required size reported */
  PPB_ERR_NOT_FOUND = -8     /* unknown ticket */
};

typedef struct ppb_ctx ppb_ctx;

/* Tile parameters: the fields of PipelineConfig used by run_tile
 * (src/IO/Parameters.jl:17-46) plus the seed of run_tile(cfg; seed).
 * Omx is the CDM-only density; the total matter density is Omx + OmB. */
typedef struct ppb_tile_params {
  double Omx, OmB, Omvac, h;
  int32_t n;
  double boxsize;
  int32_t nbuff;
  double z_out, z_max;
  int32_t ievol;
  double cenx, ceny, cenz;
  int32_t ilpt;
  int32_t ioutshear;
  int32_t wsmooth;
  /* rmax2rs > 0 (the reference's default 1.0): a peak of filter radius Rf
   * uses the first min(floor(4/3 pi (rmax2rs Rf / alatt)^3), npartmax) cells
   * of the shell list (RadialShell.jl:288-295); 0 uses the whole list */
  double rmax2rs;
  uint64_t seed;
  /* path selection: 0 = optimised path (adaptive shell truncation,
   * compensated FP32 shell sums), 1 = plain path (full spheres, FP64 shell
   * sums, unbatched transforms) */
  int32_t plain;
  int32_t reserved0;
  /* P(k) multiplier for this tile (0 means 1): a sigma8 rescale of the
   * resident table is pk_scale = (sigma8 / sigma8_table)^2 */
  double pk_scale;
  int32_t reserved[4];
} ppb_tile_params;

/* Halo output: caller-allocated record buffer.  On PPB_ERR_CAPACITY `count`
 * holds the number of records needed. */
typedef struct ppb_halo_buf {
  float* records;       /* capacity x nfields floats (host or device) */
  int64_t capacity;     /* in records */
  int64_t count;        /* out: records written */
  int32_t nfields;      /* out: 11 (ioutshear == 0) or 33 */
  float RTHLmax;        /* out: max RTHL (Mpc/h), 0 when empty (Pipeline.jl:314-318) */
  int64_t npeaks;       /* out: peak candidates found over the filter bank */
} ppb_halo_buf;

/* Serving statistics (ppb_stats_get). */
typedef struct ppb_stats {
  int64_t tiles_done;         /* requests finished (successfully or not) */
  int64_t peaks_done;
  int64_t halos_done;
  double p50_ms, p99_ms;      /* request latency, submit -> result ready */
  double tiles_per_s;         /* tiles_done / (last completion - first submit) */
  uint64_t hbm_in_use;        /* device bytes reserved by the serving slots */
  uint64_t hbm_budget;
  int32_t in_flight;          /* requests running on a slot */
  int32_t queued;             /* requests waiting for a slot or for memory */
  int32_t slots;
  int32_t failed;             /* requests that ended with an error */
} ppb_stats;

/* ---- context ------------------------------------------------------------ */
/* One context per GPU (set_cuda_device!, ext/CUDAExt.jl:3322-3325).
 * hbm_budget = 0 means 90% of the free device memory at creation. */
int32_t ppb_ctx_create(int32_t device, uint64_t hbm_budget, ppb_ctx** out);
int32_t ppb_ctx_destroy(ppb_ctx* ctx);
int32_t ppb_last_error(ppb_ctx* ctx, char* buf, size_t len);
int32_t ppb_abi_version(void);

/* ---- resident tables ---------------------------------------------------- */
/* Collapse table zvir(log10 F, e, p/e) = 1 + z_vir, Nx x Ny x Nz Float32
 * column-major, grid range(X1, X2, length=Nx) etc.; outside -> -1.
 * Replaces read_homeltab + CollapseTableInterp
 * (src/EllipsoidalCollapse/CollapseTable.jl:102-145). */
int32_t ppb_set_collapse_table(ppb_ctx* ctx, const float* tab, int32_t nx, int32_t ny, int32_t nz,
                               double x1, double x2, double y1, double y2, double z1, double z2);
/* P(k) table (k in h/Mpc, P in the reference's file convention) for the
 * log-log interpolant of load_pk (src/InitialConditions/PowerSpectrum.jl:11-30). */
int32_t ppb_set_pk_table(ppb_ctx* ctx, const double* k, const double* pk, int32_t n);
/* The collapse table with Float64 nodes (same layout and ranges as
 * ppb_set_collapse_table; replaces the resident table). */
int32_t ppb_set_collapse_table_f64(ppb_ctx* ctx, const double* tab, int32_t nx, int32_t ny, int32_t nz, double x1,
                                   double x2, double y1, double y2, double z1, double z2);

/* ---- the drop-in for run_tile ------------------------------------------ */
/* Pipeline.run_tile(cfg; seed) (src/Pipeline.jl:66-325): noise -> sqrt(P)
 * convolution -> 1LPT/2LPT -> filter bank + peak finding -> radial-shell
 * collapse -> 11/33-field records, in peak order.  Rf holds the filter radii
 * (Mpc/h, any order; sorted descending inside as Pipeline.jl:82 does).
 * Writing the .pksc file is left to the caller (ppb_write_pksc). */
int32_t ppb_run_tile(ppb_ctx* ctx, const ppb_tile_params* p, const double* Rf, int32_t nfilt,
                     ppb_halo_buf* out);

/* Same as ppb_run_tile but the timing of the device work is returned in
 * *device_ms (CUDA events on the context stream). */
int32_t ppb_run_tile_timed(ppb_ctx* ctx, const ppb_tile_params* p, const double* Rf, int32_t nfilt,
                           ppb_halo_buf* out, float* device_ms);

/* run_multitile(cfg; ntile, seed) (src/MultiTile.jl:108-418): fields on the
 * full periodic grid N = nsub ntile + 2 nbuff (nsub = n - 2 nbuff,
 * alatt = boxsize / n), the filter bank on the full grid, peaks per tile in
 * its nsub^3 core (lightcone: fcrit at the tile centre's redshift, tiles
 * beyond chi(z_max) dropped), shells per tile on the tile's own fields.
 * tiles: ntiles (it, jt, kt) triples, 1-based, in the order to process; NULL
 * (ntiles = 0) means every tile in the reference's loop order (it fastest).
 * Records are in tile order; output as ppb_run_tile. */
int32_t ppb_run_multitile(ppb_ctx* ctx, const ppb_tile_params* p, const double* Rf, int32_t nfilt, int32_t ntile,
                          const int32_t* tiles, int32_t ntiles, ppb_halo_buf* out);

/* merge_catalog(halos) (src/Merger/Merger.jl:21-78, Exclusion.jl:198-321):
 * Lagrangian exclusion in decreasing radius, then volume reduction of the
 * survivors' overlaps.  records: n x nfields (11 or 33) floats, host or
 * device; out: room for n records (host or device; may not alias records);
 * *n_out = survivors, written in input order with the reduced RTHL. */
int32_t ppb_merge_catalog(ppb_ctx* ctx, const float* records, int64_t n, int32_t nfields, float* out,
                          int64_t* n_out);

/* The fields of run_tile's first phase for params p (src/Pipeline.jl:90-140):
 * delta = generate_grf(n, P, boxsize, seed), psi = displacements_1lpt,
 * psi2 = displacements_2lpt (ilpt >= 2), lapd = irfft(k^2 delta_k)/n^3
 * (ioutshear >= 1).  Outputs are n^3 column-major Float32 (psi, psi2: three
 * consecutive components), host or device; any may be NULL. */
int32_t ppb_generate_fields(ppb_ctx* ctx, const ppb_tile_params* p, float* delta, float* psi, float* psi2,
                            float* lapd);

/* write_catalog_hdf5(path, halos, cosmo; z_max) (ext/HDF5Ext.jl:47-104;
 * stub src/PeakPatch.jl:67): the catalogue of n records (11 or 33 floats,
 * host or device) as one-dimensional Float32 datasets in the root group of
 * an HDF5 file: x, y, z, ra, dec, redshift, chi, M200m, RTHL, vx, vy, vz
 * (+ vx2, vy2, vz2, overdensity, e_v, p_v, Rf, zform for 33-field records),
 * with chi = |x| (Mpc/h), redshift from the chi -> z table up to z_max,
 * M200m = 4/3 pi 2.775e11 Om h^2 RTHL^3 (Om the total matter density),
 * (ra, dec) in radians.  Written without libhdf5 in the format's original
 * layout (superblock 0, one symbol table, contiguous storage); n = 0 writes
 * an empty file with an empty root group. */
int32_t ppb_write_catalog_hdf5(const char* path, const float* records, int64_t n, int32_t nfields, double Om,
                               double OL, double h, double z_max);

/* write_pksc (src/IO/Catalog.jl:53-94): Int32 N, Float32 RTHLmax, Float32 z_out,
 * then N x nfields Float32 (little endian). */
int32_t ppb_write_pksc(const char* path, const float* records, int64_t n, int32_t nfields,
                       float RTHLmax, float z_out);

/* ---- stub-level entry points ------------------------------------------- */
/* fill_noise_threefry! (src/InitialConditions/RandomField.jl:70-83):
 * Gaussian white noise, n^3 Float32, column-major. */
int32_t ppb_noise_threefry(ppb_ctx* ctx, float* out, int32_t n, uint64_t seed);

/* find_peaks (src/HaloFinder/PeakFind.jl:15-79) on one field; mask (Int8,
 * n^3) is read and updated.  Peaks are returned in the reference's scan order
 * (k, then j, then i).  As the reference, the scan stops after
 * max(max_peaks, 1) peaks (it tests the count after each push, :66-71), so
 * later cells are neither reported nor masked.  Outputs (capacity
 * max(max_peaks, 1)): 1-based i, j, k, ipp (int64) and delta (Float32);
 * *npeaks receives the count. */
int32_t ppb_find_peaks(ppb_ctx* ctx, const float* delta, int8_t* mask, int32_t n1, int32_t n2,
                       int32_t n3, int32_t nbuff, float fcrit, int64_t max_peaks, int64_t* pi,
                       int64_t* pj, int64_t* pk, int64_t* ipp, float* pdelta, int64_t* npeaks);

/* peak_find_tile_gpu(delta_tile, filters, fcrits, tile_masks_in, xbx, ybx,
 * zbx, alatt, nbuff, wsmooth, ioutshear) (src/PeakPatch.jl:341-366; method
 * ext/CUDAExt.jl:3068-3197): rfft(delta) once on the tile's periodic box
 * (boxsize n alatt), then for each filter in the given order smooth_field
 * with window wsmooth (0 Gaussian, 1 top-hat, 3 k^2-weighted Gaussian) and
 * find_peaks with fcrit[f] and the mask carried across filters; with
 * ioutshear >= 1 the k^2-weighted (wsmooth 3) field is sampled at each peak.
 * delta_tile: n^3 Float32 column-major; mask: n^3 Int8, read and updated.
 * Peaks come in (filter, scan order k, j, i) order, the order of the CPU
 * loop over smooth_field + find_peaks.  Outputs, capacity entries each, host
 * or device, any may be NULL: 1-based i, j, k; ipp; x = xbx + alatt (i -
 * (n+1)/2) etc.; FcRf = the smoothed delta at the peak (PeakCandidate.delta);
 * Rf of the peak's filter; d2Rf (0 without ioutshear); the 1-based filter
 * number.  *npeaks receives the count; when it exceeds capacity the call
 * returns PPB_ERR_CAPACITY and leaves the mask as it was. */
int32_t ppb_peak_find_tile(ppb_ctx* ctx, const float* delta_tile, int32_t n, const double* Rf, const double* fcrit,
                           int32_t nfilt, int8_t* mask, double xbx, double ybx, double zbx, double alatt,
                           int32_t nbuff, int32_t wsmooth, int32_t ioutshear, int64_t capacity, int32_t* pi,
                           int32_t* pj, int32_t* pk, int64_t* ipp, double* x, double* y, double* z, float* FcRf,
                           double* Rf_out, float* d2Rf, int32_t* filter, int64_t* npeaks);

/* ppb_find_peaks for callers that cannot allocate device memory at call time
 * (memory owned by another runtime's pool, or a fixed-footprint service loop
 * where cudaMalloc/cudaFree are not allowed).  No counterpart in the
 * reference: it is an addition of this library.  Same results as
 * ppb_find_peaks, but every array argument must be device memory of the
 * context's GPU, owned by the caller (npeaks is a host pointer; a buffer on
 * another GPU returns PPB_ERR_INVALID), and the call allocates nothing: its
 * scratch is a 2 MiB array built into the library, which limits the inner
 * cube to 268,435,456 cells (larger inputs return PPB_ERR_INVALID).  All
 * calls on a device share that array, so calls that overlap on the GPU race
 * and must be serialised; the first call on a device looks up the array's
 * address and should come before any stream capture. */
int32_t ppb_find_peaks_noalloc(ppb_ctx* ctx, const float* delta, int8_t* mask, int32_t n1, int32_t n2,
                               int32_t n3, int32_t nbuff, float fcrit, int64_t max_peaks, int64_t* pi,
                               int64_t* pj, int64_t* pk, int64_t* ipp, float* pdelta, int64_t* npeaks);

/* analyse_peak over a batch of peaks (src/HaloFinder/RadialShell.jl:282-891;
 * GPU stub analyse_peaks_gpu_cuda_multirf, src/PeakPatch.jl:231-253).
 * Fields are n^3 Float32 column-major (cubic grid); eta2* and lapd may be
 * NULL.  Per peak: 1-based flat index ipp, Rf (Mpc/h), ir2min, ZZon = 1+z and
 * fcrit.  nhunt is the shell radius (precompute_shells(nhunt)).  Output:
 * npk x 31 doubles per peak:
 *   0 RTHL, 1 Srb, 2-4 Sbar, 5-7 Sbar2, 8-16 strain (column-major 3x3),
 *   17-19 gradpk, 20-22 gradpkrf, 23 Fbarx, 24 e_v, 25 p_v, 26 zvir_half,
 *   27-29 gradpkf, 30 d2F.
 * The whole list is analysed (rmax2rs = 0); ppb_analyse_peaks_multirf takes
 * rmax2rs and a mask. */
int32_t ppb_analyse_peaks(ppb_ctx* ctx, const float* delta, const float* etax, const float* etay,
                          const float* etaz, const float* eta2x, const float* eta2y,
                          const float* eta2z, const float* lapd, int32_t n, int32_t nhunt,
                          int64_t npk, const int64_t* ipp, const double* Rf, const int64_t* ir2min,
                          const double* ZZon, const double* fcrit, double alatt, int32_t plain,
                          double* out);
/* ppb_analyse_peaks with a shell list per peak: peak q analyses the cells
 * with r^2 <= r2lim[q] (in cells^2; the reference's precompute_shells(R) for
 * R^2 = r2lim[q]), clipped to nhunt^2; r2lim NULL or an entry <= 0 means the
 * whole nhunt list. */
int32_t ppb_analyse_peaks_lim(ppb_ctx* ctx, const float* delta, const float* etax, const float* etay,
                              const float* etaz, const float* eta2x, const float* eta2y, const float* eta2z,
                              const float* lapd, int32_t n, int32_t nhunt, int64_t npk, const int64_t* ipp,
                              const double* Rf, const int64_t* ir2min, const double* ZZon, const double* fcrit,
                              const int32_t* r2lim, double alatt, int32_t plain, double* out);

/* analyse_peaks_gpu_cuda_multirf(delta, etax, etay, etaz, eta2x, eta2y,
 * eta2z, batches, stab, ct_table, X1, X2, Y1, Y2, Z1, Z2, alatt, ZZon; lapd,
 * mask, nbuff, growth_tables, rmax2rs, fcrit_override) (src/PeakPatch.jl:
 * 231-253; batch tuple ext/CUDAExt.jl:2327-2334): analyse_peak
 * (RadialShell.jl:282-891) over nbatch batches of peaks, one filter scale
 * each.  Batch b holds peaks boff[b] .. boff[b+1]-1 with 1-based pi, pj, pk,
 * the batch's Rf[b] (Mpc/h) and ir2min[b]; ZZon_pp / fcrit_pp give per-peak
 * redshift and fcrit (the 7-tuple batches of the lightcone) or are both NULL
 * for the scalars ZZon and fcrit (the caller resolves fcrit_override /
 * fsc_of_z(ZZon - 1) / 1.686 as the reference does).  The shell list is
 * precompute_shells(nhunt) (stab); the collapse table is the resident one
 * (ppb_set_collapse_table with the X1..Z2 ranges).  rmax2rs > 0 caps each
 * peak's list at npart = min(floor(4/3 pi (rmax2rs Rf/alatt)^3), npartmax)
 * cells.  mask (n^3 Int8, or NULL) is read and updated batch by batch: a
 * peak of batch b is skipped (no collapse) when rmax2rs > 0 and its cell's
 * mask value, as it stood before batch b, exceeds floor(Rf/alatt rmax2rs);
 * after batch b every halo of the batch sets mask = 1 over its cells within
 * RTHL in the interior nbuff+1 .. n-nbuff (the reference's GPU method reads
 * and writes the mask from concurrent threads inside a batch).  Fields and
 * per-peak arrays may be host or device memory; boff, Rf and ir2min are host
 * arrays.  out: boff[nbatch] x 31 doubles in the layout of
 * ppb_analyse_peaks. */
int32_t ppb_analyse_peaks_multirf(ppb_ctx* ctx, const float* delta, const float* etax, const float* etay,
                                  const float* etaz, const float* eta2x, const float* eta2y, const float* eta2z,
                                  const float* lapd, int32_t n, int32_t nhunt, int32_t nbatch, const int64_t* boff,
                                  const int32_t* pi, const int32_t* pj, const int32_t* pk, const double* Rf,
                                  const int64_t* ir2min, const double* ZZon_pp, const double* fcrit_pp, double ZZon,
                                  double fcrit, double alatt, int8_t* mask, int32_t nbuff, double rmax2rs,
                                  int32_t plain, double* out);

/* ---- multi-resolution tile fields ---------------------------------------
 * The MUSIC-style split of run_multitile_split (src/MultiResolution.jl:523-
 * 1236): a coarse M^3 periodic grid for the long modes plus, per tile, an
 * isolated zero-padded convolution of the Hoffman–Ribak residual noise.
 * Global fine grid N^3 with N % M == 0 (block = N / M <= 1024); tiles are
 * numbered (it, jt, kt) from 1 and cover nmesh^3 cells starting at global
 * cell (t - 1) nsub - (nmesh - nsub) / 2 (0-based, periodic in N).  P(k) is
 * the table of ppb_set_pk_table.  Fields are column-major Float32, host or
 * device. */

/* _downsample_noise (src/MultiResolution.jl:68-89): coarse cell (I, J, K) =
 * sum of the block^3 Float64 Threefry deviates of its fine cells (noise of
 * fill_noise_threefry! on the N^3 grid) in the reference's order, divided by
 * sqrt(block^3), rounded to Float32.  Bit-identical to the reference.
 * out: M^3. */
int32_t ppb_downsample_noise(ppb_ctx* ctx, int64_t N, int32_t M, uint64_t seed, float* out);

/* _generate_extended_residual (src/MultiResolution.jl:197-236): fine noise
 * minus coarse[cell's block] * Float32(1/sqrt(block^3)) on the tile's region
 * extended by nshell cells per side.  Bit-identical.
 * out: (nmesh + 2 nshell)^3. */
int32_t ppb_extended_residual(ppb_ctx* ctx, const float* coarse, int32_t M, int32_t it, int32_t jt, int32_t kt,
                              int32_t nsub, int32_t nmesh, int64_t N, uint64_t seed, int32_t nshell, float* out);

/* isolated_convolve_gpu_multi (stub src/PeakPatch.jl:280-298; CPU
 * _isolated_convolve, src/MultiResolution.jl:246-283): zero-pad the n_input^3
 * noise to (2 n_input)^3, one rfft, then per kernel multiply by
 * sqrt(P(k) dk^3 n2^3) times the kernel (DC := 0, dk = 2 pi / (n2 dx),
 * dx = boxsize_local / n), irfft, keep the n^3 region starting at nshell.
 * kernels: nkern triples (kernel_fn_id, dim1, dim2) with the ids of
 * isolated_convolve_gpu: 0 sqrt(P), 1 i k_dim1/k^2, 2 -i k_dim1/k^2,
 * 3 -k_dim1 k_dim2/k^2, 4 k^2.  out: nkern consecutive n^3 fields.
 * n_input <= 640 and nshell + n <= 2 n_input. */
int32_t ppb_isolated_convolve(ppb_ctx* ctx, const float* noise, int32_t n_input, double boxsize_local, int32_t n,
                              const int32_t* kernels, int32_t nkern, int32_t nshell, float* out);

/* interpolate_to_tile_gpu (stub src/PeakPatch.jl:329-339; CPU
 * _interpolate_to_tile / _tricubic, src/MultiResolution.jl:95-122, 156-189):
 * Catmull-Rom tricubic interpolation of the periodic M^3 coarse field at the
 * tile's fine cells.  Bit-identical.  out: nmesh^3. */
int32_t ppb_interpolate_to_tile(ppb_ctx* ctx, const float* coarse, int32_t it, int32_t jt, int32_t kt, int32_t nsub,
                                int32_t nmesh, int64_t N, int32_t M, float* out);

/* compute_2lpt_gpu (stub src/PeakPatch.jl:300-316; CPU block
 * src/MultiResolution.jl:804-831): tile-local periodic 2LPT of delta_tile,
 * src2 = delta^2/2 - sum_a phi_aa^2/2 - sum_{a<b} phi_ab^2, psi2_d =
 * irfft(-i k_d/k^2 rfft(src2)), with _apply_kernel_inplace!'s zeroing of the
 * DC mode and the Nyquist planes.  psi2: 3 consecutive n^3 fields. */
int32_t ppb_compute_2lpt(ppb_ctx* ctx, const float* delta_tile, int32_t n, double boxsize_local, float* psi2);

/* compute_laplacian_gpu (stub src/PeakPatch.jl:318-327; CPU
 * src/MultiResolution.jl:835-846): irfft(k^2 rfft(delta_tile)) with the same
 * zeroing (no extra 1/n^3, unlike run_tile's lapd).  lapd: n^3. */
int32_t ppb_compute_laplacian(ppb_ctx* ctx, const float* delta_tile, int32_t n, double boxsize_local, float* lapd);

/* The coarse phase of run_multitile_split (src/MultiResolution.jl:617-667)
 * on the M^3 coarse noise, each field an irfft of _periodic_convolve!
 * (:286-309) of its rfft in a box of side boxsize_full: delta (M^3), psi
 * (3 M^3, 1LPT kernels), psi2 (3 M^3, ilpt >= 2: the trace-identity source
 * convolved with sqrt(P) and the 2LPT kernel, as the reference does) and
 * lapd (M^3, ioutshear >= 1).  Any output may be NULL. */
int32_t ppb_coarse_fields(ppb_ctx* ctx, const float* coarse_noise, int32_t M, double boxsize_full, int32_t ilpt,
                          int32_t ioutshear, float* delta, float* psi, float* psi2, float* lapd);

/* run_multitile_split(cfg; ntile, seed, coarse_factor, coarse_grid,
 * use_gpu=true) (src/MultiResolution.jl:523-1236): N = nsub ntile + 2 nbuff
 * (nsub = n - 2 nbuff, alatt = boxsize / n); coarse grid M as
 * ppb_split_coarse_grid; coarse noise and coarse delta / psi on M^3; per tile
 * the split fields (ppb_extended_residual -> ppb_isolated_convolve with
 * kernels delta, psi_x, psi_y, psi_z -> plus ppb_interpolate_to_tile of the
 * coarse fields; ppb_compute_2lpt and ppb_compute_laplacian of the tile's
 * delta), then the filter bank, peaks, shells and records on the tile's own
 * n^3 grid as run_tile does, with the tile centre's position and (ievol = 1)
 * the fcrit of its redshift; tiles beyond chi(z_max) dropped.  tiles as
 * ppb_run_multitile.  Records in tile order (no merge), output as
 * ppb_run_tile.  n <= 640. */
int32_t ppb_run_multitile_split(ppb_ctx* ctx, const ppb_tile_params* p, const double* Rf, int32_t nfilt,
                                int32_t ntile, int32_t coarse_factor, int32_t coarse_grid, const int32_t* tiles,
                                int32_t ntiles, ppb_halo_buf* out);

/* The coarse grid M of run_multitile_split (src/MultiResolution.jl:592-612):
 * coarse_grid when > 0, else ntile coarse_factor when > 0, else the divisor m
 * of N in [2, N/2] whose block N/m is closest to n/3 (the smallest such m).
 * Returns M (0 when no divisor exists) or PPB_ERR_INVALID. */
int32_t ppb_split_coarse_grid(int32_t n, int32_t nbuff, int32_t ntile, int32_t coarse_factor, int32_t coarse_grid);

/* ---- memory helpers ----------------------------------------------------- */
/* Page-locked host memory (fast, asynchronous copies of records) and device
 * memory on the context's GPU, for callers that have no CUDA runtime of
 * their own (a Julia or Python host).  Free with the matching call. */
int32_t ppb_alloc_host(ppb_ctx* ctx, size_t bytes, void** out);
int32_t ppb_free_host(ppb_ctx* ctx, void* p);
int32_t ppb_alloc_device(ppb_ctx* ctx, size_t bytes, void** out);
int32_t ppb_free_device(ppb_ctx* ctx, void* p);

/* ---- serving ------------------------------------------------------------ */
/* A serving loop over the same tables (no reference counterpart: the
 * reference runs one run_tile at a time).  Requests of any grid size, seed
 * and cosmology are queued by ppb_submit and run on `slots` execution slots,
 * each with its own CUDA stream and buffers, so that tiles of different
 * requests overlap on the device.  A request is started as soon as a slot is
 * idle and the HBM budget of the context admits its footprint (fields,
 * transforms, peak and shell buffers of its grid size); a request that could
 * never fit fails with PPB_ERR_ADMISSION.  The collapse and P(k) tables stay
 * resident and are shared; ppb_set_* waits for the runs in flight.
 * Results are the same as ppb_run_tile's for the same parameters.
 *
 * ppb_serve_config sets the number of slots (1..32, default 4) before the
 * first submit.  ppb_submit copies params and Rf and returns a ticket.
 * ppb_wait blocks up to timeout_ms (< 0: no limit) for the ticket's result and
 * copies the records into `out` like ppb_run_tile (PPB_ERR_TIMEOUT leaves the
 * request in place; PPB_ERR_CAPACITY reports the count needed and keeps the
 * result for another wait).  A failed request returns its error code and
 * message.  Each ticket is waited for once. */
int32_t ppb_serve_config(ppb_ctx* ctx, int32_t slots);
int32_t ppb_submit(ppb_ctx* ctx, const ppb_tile_params* p, const double* Rf, int32_t nfilt, uint64_t* ticket);
int32_t ppb_wait(ppb_ctx* ctx, uint64_t ticket, int32_t timeout_ms, ppb_halo_buf* out);
int32_t ppb_stats_get(ppb_ctx* ctx, ppb_stats* out);
/* Clears the latency record and counters of ppb_stats (not the queue). */
int32_t ppb_stats_reset(ppb_ctx* ctx);

/* ---- timing helpers ----------------------------------------------------- */
/* Named CUDA events on the context stream (slot 0..15). */
int32_t ppb_event_record(ppb_ctx* ctx, int32_t slot);
int32_t ppb_event_elapsed(ppb_ctx* ctx, int32_t a, int32_t b, float* ms);
int32_t ppb_synchronize(ppb_ctx* ctx);
/* Count of kernel launches issued by this library since context creation. */
int32_t ppb_launch_count(ppb_ctx* ctx, int64_t* count);
/* Shell-stage statistics of the last run: in-bounds cell visits, the five
 * dump-reason counters of src/HaloFinder/RadialShell.jl:15-34 (premask,
 * no_fcrit, m0_one, no_collapse, rthl_neg) and the stage's device time. */
int32_t ppb_last_shell_stats(ppb_ctx* ctx, int64_t* visits, int64_t* dumps5, float* ms);
/* All 16 raw shell-stage counters of the last run: [0] cell visits,
 * [1..5] dump reasons as above, [6] profile reads beyond the gathered shells
 * (must be 0), [7] SPH-table overruns (the reference raises there),
 * [8] invalid peak inputs, [9] collapse-walk steps evaluated, others reserved. */
int32_t ppb_shell_counters(ppb_ctx* ctx, int64_t* out16);
/* Device time (ms) of the shell stage's four kernels in the last run:
 * [0] gather, [1] collapse walk, [2] zvir_half, [3] d2F; *rows = profile
 * rows written (24 doubles each), *batches = peak batches the stage ran in. */
int32_t ppb_last_shell_times(ppb_ctx* ctx, float* ms4, int64_t* rows, int32_t* batches);
/* ---- collapse-table generation ------------------------------------------ */
/* make_table (src/EllipsoidalCollapse/CollapseTable.jl:33-52) with the RK4
 * solver (EllipsoidParams(cosmo; solver = :rk4), evolve_ellipse_full,
 * src/EllipsoidalCollapse/EllipsoidalCollapse.jl:518-624), one FP64
 * integration per node on the GPU.  Fields mirror CosmologyParams (Om is the
 * total matter density), CollapseTableParams and the EllipsoidParams
 * defaults (iforce_strat 4, ivir_strat 2, fcoll 0.01 / 0.171 / 0.171,
 * tfac 0.01, nstepmax 10000, zinit_fac 20; Carlson RD shape integrals). */
typedef struct ppb_table_params {
  double Om, OB, OL, h;
  int32_t Nx, Ny, Nz;            /* nodes along log10 F, e_v, p_v / e_v (50, 20, 20) */
  int32_t iforce_strat;          /* 0, 1, 3, 4, 5 or 6 */
  int32_t ivir_strat;            /* 1 or 2 */
  int32_t nstepmax;
  double X1, X2;                 /* log10 F range (log10 1.5, log10 8) */
  double Y1, Y2;                 /* e_v range (0, 0.5) */
  double Z1, Z2;                 /* p_v / e_v range (-1 + 1e-4, 1 - 1e-4) */
  double fcoll_1, fcoll_2, fcoll_3, tfac, zinit_fac;
  int32_t reserved[4];
} ppb_table_params;
/* Computes the Nx x Ny x Nz table of 1 + z_vir (-1: no collapse) in double
 * precision, column-major (i fastest), into `out` (host or device, may be
 * null) and, with install = 1, makes it the context's collapse table rounded
 * to Float32 (the reference's table) or, with install = 2, with Float64
 * nodes.  ppb_last_table_stats reports the device time and the RK4 steps. */
int32_t ppb_make_collapse_table(ppb_ctx* ctx, const ppb_table_params* p, double* out, int32_t install);
int32_t ppb_last_table_stats(ppb_ctx* ctx, float* ms, int64_t* steps);

/* ---- launch options and the autotuner ------------------------------------ */
/* Context options (no reference counterpart).
 *  PPB_OPT_GRAPHS     1 (default): the fields, the filter bank and each
 *                     shell-stage sub-batch (with a multi-tile run's
 *                     per-tile field windows) are recorded into CUDA graphs,
 *                     updated in place from one call to the next and
 *                     launched whole; 0: the same kernels launched one by one.
 *  PPB_OPT_AUTOTUNE   1 (default): the first shell stage of each kind of
 *                     batch (grid size, shell list, arithmetic, truncation,
 *                     per-peak limits, walk length class) with at least
 *                     PPB_OPT_TUNE_MIN_PEAKS peaks times the gather-order
 *                     bricks (4, 8, 16, 32 cells, list order) and the
 *                     collapse kernels (1, 2, 4 threads per peak, lane
 *                     queues) and keeps
 *                     the fastest; 0: defaults (8-cell bricks, width by
 *                     batch size); setting 2 clears the table.
 *                     Results do not depend on the choice.
 *  PPB_OPT_TUNE_MIN_PEAKS  smallest batch that is tuned (default 16384).
 *  PPB_OPT_BRICK_SHIFT     fixes the gather-order brick over the tuner's
 *                     choice: 2..5 (bricks of 4..32 cells), -1 list order,
 *                     -2 (default) the tuner's choice.
 *  PPB_OPT_COLLAPSE_THREADS  fixes the collapse kernel: 1, 2 or 4 threads
 *                     per peak, 8 one thread per peak with lane work queues,
 *                     0 (default) the tuner's choice.
 *  PPB_OPT_COLLAPSE_ORDER  the order the collapse kernels take the peaks
 *                     in: 1 by descending crossing shell m0 (similar walks
 *                     share a warp, the longest start first; a key kernel
 *                     and a radix sort after the gather), 0 list order, -1
 *                     (default) the tuner's choice (list order for batches
 *                     below PPB_OPT_TUNE_MIN_PEAKS).  Same records.
 *  PPB_OPT_GATHER_TEX  1: the shell gather fetches its records through a
 *                     texture object over the record array (the texture
 *                     pipe, beside the load/store pipe; grids with 2 n^3
 *                     float4 within the device's linear-texture limit);
 *                     0: 256-bit loads; -1 (default): the tuner times both
 *                     and keeps the faster (the texture pipe for batches it
 *                     does not tune).  Same records.
 *  PPB_OPT_GATHER_RING  1: the shell gather stages its records through
 *                     per-lane shared-memory rings filled by TMA
 *                     (tile::gather4 bulk tensor copies, two stages, bounded
 *                     mbarrier waits); 0 (default): 256-bit loads straight
 *                     from global memory.  Same records either way; the
 *                     staged form is slower on B200 (the TMA unit serialises
 *                     the 128-byte gathers) and is kept for comparison.
 *  PPB_OPT_FUSED_X    the filter bank's x pass fused with the peak search
 *                     (grid sizes 64 J, J <= 8, one window over the grid):
 *                     -1 (default) with the k^2-weighted twin (ioutshear)
 *                     for J = 3, 5, 6, 7 (where the 3-D C2R is slowest),
 *                     1 wherever supported, 0 never (full 3-D C2R +
 *                     separate search).
 *                     The peaks agree up to FP32 transform rounding.
 * Read-only (ppb_get_option, summed over the context's slots):
 *  PPB_OPT_GRAPH_LAUNCHES, PPB_OPT_GRAPH_INSTANTIATIONS, PPB_OPT_GRAPH_UPDATES. */
enum {
  PPB_OPT_GRAPHS = 1,
  PPB_OPT_AUTOTUNE = 2,
  PPB_OPT_TUNE_MIN_PEAKS = 3,
  PPB_OPT_BRICK_SHIFT = 4,
  PPB_OPT_COLLAPSE_THREADS = 5,
  PPB_OPT_FUSED_X = 6,
  PPB_OPT_GATHER_RING = 7,
  PPB_OPT_COLLAPSE_ORDER = 8,
  PPB_OPT_GATHER_TEX = 10,
  PPB_OPT_GRAPH_LAUNCHES = 16,
  PPB_OPT_GRAPH_INSTANTIATIONS = 17,
  PPB_OPT_GRAPH_UPDATES = 18
};
int32_t ppb_set_option(ppb_ctx* ctx, int32_t option, int64_t value);
int32_t ppb_get_option(ppb_ctx* ctx, int32_t option, int64_t* value);

/* One autotuned shell-stage configuration. */
typedef struct ppb_tune_entry {
  int32_t n, nshell;          /* grid size, distinct r^2 of the shell list */
  int32_t comp, adaptive;     /* compensated FP32 sums, adaptive truncation */
  int32_t limited;            /* per-peak shell limits (ppb_analyse_peaks_lim) */
  int32_t brick_shift;        /* chosen order brick: 2^brick_shift cells, -1 = list order */
  int32_t collapse_threads;   /* chosen collapse width, 0 = by batch size */
  int32_t long_walk;          /* batches after ones with > 8 collapse-walk steps per peak (lightcone) */
  int64_t npk;                /* peaks of the batch the candidates were timed on */
  float gather_ms[5];         /* gather kernel: bricks of 4, 8, 16, 32 cells, list order */
  float collapse_ms[4];       /* collapse kernel: 1, 2, 4 threads per peak, lane work queues (8) */
  int32_t collapse_order;     /* chosen: 1 = peaks by descending crossing shell, 0 = list order */
  float collapse_ordered_ms[4];   /* the collapse widths with that order */
  int32_t gather_tex;         /* chosen: 1 = records through the texture pipe, 0 = 256-bit loads */
  float gather_plain_ms;      /* the chosen order with 256-bit loads (0 when no texture was available) */
} ppb_tune_entry;
/* Copies up to `cap` entries; *n = the number of entries held. */
int32_t ppb_tune_entries(ppb_ctx* ctx, ppb_tune_entry* out, int32_t cap, int32_t* n);

/* Per-stage device times (ms) of the last ppb_run_tile_timed call:
 * [0] fields, [1] filter bank + peaks, [2] shell analysis, [3] records. */
int32_t ppb_last_stage_ms(ppb_ctx* ctx, float* ms4);

#ifdef __cplusplus
}
#endif
#endif /* PPB_H */
