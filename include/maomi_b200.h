/*
 * maomi_b200.h -- C ABI of the B200-native MaoMi optical stage.
 *
 * Plain C: device pointers, sizes and a cudaStream_t (passed as void*).  No
 * entry point allocates device memory; buffers and workspaces belong to the
 * caller (query sizes with the *_workspace_size functions).  Every entry
 * point returns MM_OK (0) or a negative status and records a message that
 * mm_last_error() returns (thread-local).  Kernels run on the given stream
 * and the calls do not synchronise unless stated.
 *
 * Each declaration names the reference interface it replaces (paths relative
 * to the MaoMi 0.8.0b1 source tree).
 */
#ifndef MAOMI_B200_H
#define MAOMI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  MM_OK = 0,
  MM_ERR_ARGUMENT = -1,   /* shape, size or range error (Python: ValueError) */
  MM_ERR_CUDA = -2,       /* CUDA runtime error (Python: RuntimeError)       */
  MM_ERR_TIMEOUT = -3,    /* a bounded device wait gave up (RuntimeError)    */
  MM_ERR_NONFINITE = -4,  /* non-finite input rejected (ValueError)          */
  MM_ERR_UNSUPPORTED = -5 /* no kernel for this size (ValueError)            */
};

/* Library version (major*10000 + minor*100 + patch). */
int mm_version(void);

/* Message of the last failing call on this host thread ("" if none). */
const char* mm_last_error(void);

/* 1 if the current device is an sm_100 part the library was built for. */
int mm_device_supported(void);

/* sizeof of a descriptor struct of this header, by its type name
   ("mm_stage_plan", ...; 0 for an unknown name): lets a binding check its
   own record layout against the library's.  No counterpart in the
   reference, whose kernels take no structs. */
size_t mm_struct_size(const char* name);

/* Kernels launched by this library since it was loaded (all threads). */
unsigned long long mm_launch_count(void);

/* ------------------------------------------------------------------------
 * Screen gather: dst[b,z,x,y] = src[z, off[b,0]+x, off[b,1]+y] * edge[x*N+y]
 * Replaces gather_screens, maomi/backends/cuda/optical_kernels.cu:3-12
 * (bound by gather(), maomi/backends/cuda/native.py:19-24).
 */
int mm_gather_screens(const void* src /* float2 (Z,H,W) */, const float* edge /* (N,N) */,
                      const int32_t* offsets /* (B,2) */, void* dst /* float2 (B,Z,N,N) */,
                      int B, int Z, int H, int W, int N, void* stream);

/* ------------------------------------------------------------------------
 * Sparse separable power resample: out[b,x,y,z] = scale*axial[z] *
 *   sum_i wx[x,i] sum_j wy[y,j] |field[b,z,ix[x,i],iy[y,j]]|^(2*order)
 * Replaces resample_power, maomi/backends/cuda/optical_kernels.cu:14-38
 * (bound by ResamplePlan.__call__, maomi/backends/cuda/native.py:68-105).
 */
int mm_resample_power(const void* field /* float2 (B,Z,H,W) */, const int32_t* ix, const float* wx,
                      const int32_t* iy, const float* wy, const float* axial /* (Z) */,
                      float* out /* (B,X,Y,Z) */, int B, int Z, int H, int W, int X, int Y,
                      int KX, int KY, int order, float scale, void* stream);

/* ------------------------------------------------------------------------
 * MATLAB v4 Green-function evaluation in FP64:
 *   out[q,c] = sum_i g(|query_q - p_i|^2) * coef[i,c],  g(r2) = r2*(0.5*log(r2)-1), g(0)=0
 * Replaces green_apply, maomi/backends/cuda/interpolation.cu:3-19 (bound by
 * evaluate_v4, maomi/backends/cuda/interpolation.py:17-38).  Any ncoef >= 1.
 */
int mm_green_apply(const double* points /* (n,2) */, const double* coef /* (n,ncoef) */,
                   const double* queries /* (m,2) */, double* out /* (m,ncoef) */,
                   int n, int m, int ncoef, void* stream);

/* Dense v4 system matrix G[i,j] = |p_i-p_j|^2 (log|p_i-p_j| - 1), G[i,i] = 0
 * (the matrix solved in maomi/numerics.py:122-129). */
int mm_green_matrix(const double* points /* (n,2) */, double* G /* (n,n) */, int n, void* stream);

/* mm_green_apply_grid for points at integer coordinates in
 * [px_min, px_max] x [py_min, py_max]: every query-point offset is a half
 * integer, so g is tabulated once per offset into `table`
 * ((X - px_min + px_max) * (Y - py_min + py_max) doubles) and the sums read it;
 * same point order and FMA chain as mm_green_apply_grid (identical results). */
int mm_green_apply_grid_table(const double* points, const double* coef, double* out, int n, int X, int Y, int ncoef,
                              int px_min, int px_max, int py_min, int py_max, double* table, size_t table_bytes,
                              void* stream);

/* The v4 system of points on a full nx x ny lattice symmetric under both
 * axis reflections (the fixed site lattice, maomi/fixed.py:15-33) in the basis
 * of even/odd reflection pairs: four independent symmetric blocks, parity
 * b = 2*(x odd) + (y odd), each padded to m x m with the identity
 * (m >= ceil(nx/2)*ceil(ny/2)).  lattice[i*ny + j] = index of the point at
 * the i-th x and j-th y coordinate.  Same linear system as mm_green_matrix. */
int mm_green_blocks(const double* points, const int32_t* lattice, int nx, int ny, int m,
                    double* blocks /* (4,m,m) */, void* stream);
/* In-place x <- A^-1 x for `batch` column-major m x m LU factorisations (unit
 * lower L, U, 1-based LAPACK pivots, as from getrf) with nrhs right-hand
 * sides each (x: (batch, m, nrhs)); one CTA per system (the parity blocks of
 * the v4 solve). */
int mm_lu_solve_batched(const double* lu, const int32_t* pivots, int batch, int m, int nrhs, double* x, void* stream);

/* Parity transform of v4 right-hand sides / solutions: inverse = 0 maps
 * values (n,ncoef) to block components (4,m,ncoef); inverse = 1 maps block
 * solutions (4,m,ncoef) back to coefficients (n,ncoef). */
int mm_v4_parity(const int32_t* lattice, int nx, int ny, int m, int ncoef, int inverse, const double* in,
                 double* out, void* stream);

/* v4 evaluation on a regular pixel grid (queries (i+0.5, j+0.5), i<X, j<Y),
 * the mask-assembly case of maomi/fixed.py:141-144; out is (X,Y,ncoef). */
int mm_green_apply_grid(const double* points, const double* coef, double* out,
                        int n, int X, int Y, int ncoef, void* stream);

/* ------------------------------------------------------------------------
 * Phase preparation: screens[z,x,y] = exp(1j * resize(raw, ss)[x,y,z] * scale)
 * with resize = separable index/weight tables (MATLAB imresize bicubic).
 * Replaces the phase preparation of maomi/backends/cuda/batched.py:52-60
 * (and optics.py:238-249 with numerics.py:15-39).  raw is (H,W,Z) float32
 * (XY-major, Z fastest as the reference's arrays); tables are (Ho,KX),(Wo,KY).
 */
int mm_phase_prepare(const float* raw, int H, int W, int Z,
                     const int32_t* ix, const float* wx, int Ho, int KX,
                     const int32_t* iy, const float* wy, int Wo, int KY,
                     float scale, void* screens /* float2 (Z,Ho,Wo) */,
                     float* scratch /* float (Ho,W,Z) when KX>1 or KY>1, else NULL */, void* stream);

/* ------------------------------------------------------------------------
 * Gaussian pupil with aperture, focusing phase and optional Zernike / custom
 * phase, evaluated in FP64 and rounded to complex64.
 * Replaces maomi.optics.pupil, maomi/optics.py:90-117 with
 * maomi/_optical_math.py:232-296.
 */
typedef struct {
  int n;                 /* grid points per axis                                */
  double pitch;          /* grid pitch D1 (m)                                    */
  double beam_radius;    /* Gaussian 1/e radius `rad` (m)                        */
  double aperture;       /* objective aperture radius `objrad` (m)               */
  double k;              /* wavenumber 2*pi*n/lambda (1/m)                       */
  double focal_length;   /* fl (m)                                               */
  int nmodes;            /* Zernike modes (0 = none)                             */
  const double* mode_coef;   /* host: per mode, weight*lambda (m) times norm      */
  const int* mode_m;         /* host: azimuthal order                             */
  const int* mode_cos;       /* host: 1 = cos(m t), 0 = sin(m t) (m>0)            */
  const int* mode_nterms;    /* host: radial terms per mode                       */
  const double* term_coef;   /* host: radial coefficients (concatenated)          */
  const int* term_pow;       /* host: radial powers (concatenated)                */
  const float* custom_phase; /* device (Hc,Wc) radians or NULL                    */
  int custom_h, custom_w;
  double custom_radius;      /* aperture radius the custom phase spans (m)        */
  double custom_scale;       /* 1 (radians) or 2*pi (waves)                       */
} mm_pupil_desc;

int mm_pupil(const mm_pupil_desc* desc, void* out /* float2 (n,n) */,
             double* scratch /* (n*n + 2*1024) doubles */, void* stream);

/* ------------------------------------------------------------------------
 * Base field: pupil -> tissue top by the scaled two-plane Fresnel step
 * (pitch d1 -> d2), then unit L2 norm.  Chirp phases in FP64.
 * Replaces the base computation of maomi/backends/cuda/batched.py:43-51
 * (maomi/numerics.py:156-210 with two planes; maomi/optics.py:223-231).
 */
typedef struct {
  int n;
  double d1, d2;          /* source / destination pitch (m)                       */
  double dz;              /* propagation distance (m)                             */
  double lambda_medium;   /* wavelength / n_r (m)                                 */
  const float* edge1d;    /* device: 1-D edge window (n)                          */
} mm_base_desc;

int mm_base_field(const mm_base_desc* desc, const void* pupil /* float2 (n,n) */,
                  void* out /* float2 (n,n) */, void* work /* float2 (n,n) */,
                  double* scratch /* 1024 doubles */, void* stream);

/* ------------------------------------------------------------------------
 * Fused per-site split-step propagation (stages A, B, C), screens applied
 * from the phase volumes at each site's offset, saved planes reduced in the
 * same pass: focal |E|^(2*order) crops, top/bottom tail images and profiles.
 * Replaces the hot loop of OpticalPlan.evaluate,
 * maomi/backends/cuda/batched.py:157-235 (and the per-site loop of
 * maomi/optics.py:259-340).
 */
typedef struct {
  int size;                /* window of this stage (n for A and C, n2 for B)      */
  int steps;               /* propagation steps = screens of this stage           */
  const void* screens;     /* float2 (steps, vol_h, vol_w) phase volume           */
  int vol_h, vol_w;
  const float* edge1d;     /* (size) edge window axis                              */
  const void* kernels;     /* float2 (steps, size): per-step 1-D transfer function
                              in FFT order with 1/size folded in                   */
} mm_stage_desc;

typedef struct {
  mm_stage_desc stage[3];  /* A, B, C                                             */
  const void* base;        /* float2 (n,n) field entering stage A                 */
  int n, n2;
  int order;               /* photon order 1..3                                   */
  int cut;                 /* first saved plane of stage A (top tail)             */
  int focal_x0, focal_y0, focal_h, focal_w;  /* focal crop inside the n2 window   */
  const float* tail_weight[2]; /* per saved plane: trapezoid*axial (top, bottom)   */
  /* outputs */
  float* focal;            /* (P, steps_B, focal_h, focal_w) |E|^(2*order)        */
  float* tail_image[2];    /* per_site: (P,n2,n2); else (slots,n2,n2) running sums */
  int tail_per_site;
  double* tail_profile[2]; /* (P, planes) sum over pixels of |E|^(2*order);
                              zeroed by the call                                  */
  const int32_t* offsets;  /* (P,2) window offsets on the screen lattice          */
  int nsites;
  int precision;           /* arithmetic of the radix-2 line transforms: FP32,
                              FP64 (butterflies, twiddles and filter in FP64),
                              MIXED (forward FP32, inverse FP64), COMPENSATED
                              (FP32 butterflies, every DFT rotation constant
                              carried as a hi + lo pair of floats) or
                              COMPENSATED_FULL (the twiddle tables too); the
                              field is stored complex64 in every mode             */
  int reserve_sms;         /* persistent schedule: CTAs that start on SM ids below
                              this count leave at once, so work queued on other
                              streams (e.g. the v4 factorisation) runs there
                              while the sites propagate; 0 = use every SM         */
  /* fault drill for the bounded dependency wait (leave both 0 in production):
     hold_site = s + 1 makes site s's first item wait for a counter value that
     is never published, and spin_limit (> 0) replaces the default bound of
     that wait (persistent schedule); the call then returns MM_ERR_TIMEOUT
     with every CTA exited                                                    */
  int hold_site;
  long long spin_limit;
} mm_stage_plan;

enum {
  MM_PRECISION_FP32 = 0,
  MM_PRECISION_FP64 = 1,
  MM_PRECISION_MIXED = 2,
  MM_PRECISION_COMPENSATED = 3,
  MM_PRECISION_COMPENSATED_FULL = 4
};

enum { MM_SCHEDULE_PERSISTENT = 0, MM_SCHEDULE_BATCHED = 1 };

/* Bytes of workspace mm_propagate_sites needs for `slots` sites in flight. */
size_t mm_propagate_workspace_size(const mm_stage_plan* plan, int slots, int schedule);

/* Propagate every site of the plan.  schedule: MM_SCHEDULE_PERSISTENT runs one
 * persistent launch fed by a device work queue (slots sites in flight);
 * MM_SCHEDULE_BATCHED launches each segment for `slots` sites at a time.
 * If tail_per_site is 0 the tail images must be zeroed by the caller before
 * the first call (they accumulate).  Synchronises the stream only to read
 * the device error flag when check != 0. */
int mm_propagate_sites(const mm_stage_plan* plan, int schedule, int slots, void* workspace,
                       size_t workspace_bytes, int check, void* stream);

/* The check of mm_propagate_sites on its own: synchronise the stream and read
 * the device error flag of a propagation that ran with check = 0 in
 * `workspace` (same plan, schedule and slots), for example inside a replayed
 * CUDA graph, where the call itself cannot synchronise.  Returns
 * MM_ERR_ARGUMENT for out-of-range site windows, MM_ERR_TIMEOUT for a
 * dependency wait that ran out. */
int mm_propagate_status(const mm_stage_plan* plan, int schedule, int slots, const void* workspace, void* stream);

/* Propagation for callers that cannot allocate device memory (no counterpart
 * in the reference).  Same work and outputs as mm_propagate_sites, with the
 * workspace taken from a fixed 32 MiB device array inside the library instead
 * of a caller buffer: hosts that reserve the whole device heap for their own
 * pool, or code that must not call cudaMalloc once running, can still
 * propagate.  Plans needing more scratch than the array holds (at n = n2 = 256,
 * more than 31 sites in flight) are rejected with MM_ERR_ARGUMENT.  The first
 * call on a device looks up the array's address with that device current;
 * make it before any stream capture.  All calls share the array (it keeps the
 * last call's contents); calls that overlap on the GPU race, so serialise
 * them.  Calls no cudaMalloc or cudaFree. */
int mm_propagate_sites_noalloc(const mm_stage_plan* plan, int schedule, int slots, int check, void* stream);

/* ------------------------------------------------------------------------
 * Independent propagation items of one window size (uneven depths) in one
 * persistent launch: item i propagates field_in through steps[i] screens
 * exp(1j*phase) (times an optional separable edge window), one step being
 * u <- IDFT2(Q * DFT2(u * screen)) with a 1-D transfer function `kernel`
 * applied along both axes.  Generalises the split-step loop of
 * maomi/numerics.py:189-206 (constant pitch) to a device work queue of
 * many items; the reference propagates such items one call at a time.
 * Items are processed in waves of `slots` (sort them by depth); the schedule
 * tables come from the caller (see maomi_b200/items.py).
 */
typedef struct {
  int n;                       /* window: 64, 128, 256 or 512                     */
  int nitems;
  int slots;                   /* items in flight (one wave)                      */
  int waves;
  long long total_items;       /* queue length = wave_items[waves]                */
  const int32_t* steps;        /* device (nitems)                                 */
  const int64_t* phase_offset; /* device (nitems): float offset of each (steps,n,n) stack */
  const float* phase;          /* device: flat phase stacks (radians)             */
  const void* field_in;        /* device float2 (n,n)                             */
  void* field_out;             /* device float2 (nitems,n,n)                      */
  const void* kernel;          /* device float2 (n): FFT order, 1/n folded in      */
  const float* edge1d;         /* device (n) or NULL                              */
  const int64_t* wave_items;   /* device (waves+1): first queue item of each wave */
  const int32_t* wave_levels;  /* device (waves): segments per wave (max steps+1) */
  const int32_t* slot_base;    /* device (waves*slots): counter before each wave  */
  int precision;               /* MM_PRECISION_*                                  */
  int shape;                   /* CTA shape: 0 default radices, 1 wider per thread */
} mm_item_class;

/* Line blocks per segment for window n and CTA shape (for the schedule). */
int mm_items_blocks(int n, int shape);
size_t mm_propagate_items_workspace_size(const mm_item_class* c);
int mm_propagate_items(const mm_item_class* c, void* workspace, size_t workspace_bytes, int check, void* stream);

/* ------------------------------------------------------------------------
 * Focal PSF finalisation: psf[p,x,y,z] = scale*axial[z] *
 *   sum_i wx[x,i] sum_j wy[y,j] focal[p,z,ix[x,i],iy[y,j]]
 * from the focal |E|^(2*order) crops (sparse resample tables as ResamplePlan
 * builds them), plus per-site energies (FP64 sums) and, when psf_sum and
 * psf_abs_sum are given, the site sums of psf and |psf| (FP64).  Replaces the
 * focal ResamplePlan call of maomi/backends/cuda/batched.py:194-200 and the
 * reductions of maomi/fixed.py:126,153-154.  psf may be NULL (energies only).
 * All four tables NULL: identity resample (ss = 1; X == H, Y == W), run as a
 * tiled transpose of the crops.
 */
int mm_focal_finalize(const float* focal /* (P,Z,H,W) */, const int32_t* ix, const float* wx, int KX,
                      const int32_t* iy, const float* wy, int KY, const float* axial /* (Z) */, float scale,
                      int P, int Z, int H, int W, int X, int Y,
                      float* psf /* (P,X,Y,Z) */, double* energies /* (P) */,
                      double* psf_sum /* (X,Y,Z) */, double* psf_abs_sum /* (X,Y,Z) */, void* stream);

/* Tail image finalisation: out[x,y] = scale * (Rx (sum_s img_s) Ry^T)[x,y]
 * with dense float32 resample matrices (the convmask mean of
 * maomi/fixed.py:181 with batched.py:220-223); scratch holds H*W doubles. */
int mm_tail_finalize(const float* images /* (S,H,W) */, int S, int H, int W,
                     const float* rx /* (X,H) */, const float* ry /* (Y,W) */, int X, int Y,
                     double scale, double* out /* (X,Y) */, double* scratch, void* stream);

/* Per-image sparse resample: out[s,x,y] = scale * sum wx*wy*in[s,ix,iy]
 * (the per-site tail images of batched.py:220-223). */
int mm_resample_images(const float* in /* (S,H,W) */, int S, int H, int W, const int32_t* ix, const float* wx,
                       int KX, const int32_t* iy, const float* wy, int KY, int X, int Y, float scale,
                       float* out /* (S,X,Y) */, void* stream);

/* ------------------------------------------------------------------------
 * Scattering-field generation (the stage's raw A/B/C inputs).
 * Replaces masked_3DGP_test, maomi/_optical_math.py:20-67, and the field
 * loop of prepare_fields, maomi/optics.py:145-196.  One Gaussian-process
 * draw is mm_gp_spectrum, an inverse 3-D DFT normalised by 1/N (complex64),
 * then mm_gp_finish.  Grids are C-ordered (nx, ny, nz).
 */

/* spec[x,y,z] = (re + i im)[s] * S[s], s = ((x + nx/2) % nx, (y + ny/2) % ny,
 * (z + nz/2) % nz) (ifftshift), S = sqrt(sum_k prod_l[k] (kx ky kz)^2 w2[k]),
 * kx = exp(-g2x[sx] * l2[3k]) (and y, z likewise).  g2x/g2y/g2z: the squared
 * linspace(-pi/2, pi/2, n) grids; l2: squared scales (nscales, 3); prod_l:
 * l_x l_y l_z; w2: squared weights; noise_re/noise_im: (nx,ny,nz) float32;
 * spec: complex64 (nx,ny,nz).  All device pointers. */
int mm_gp_spectrum(int nx, int ny, int nz, const float* g2x, const float* g2y, const float* g2z, int nscales,
                   const float* l2, const float* prod_l, const float* w2, const float* noise_re,
                   const float* noise_im, void* spec, void* stream);

/* out[x,y,z] = scale * Re(y[ifftshift(x,y,z)]), times `first` on z = 0 and
 * `last` on z = nz-1 (the partial-slab factors of optics.py:167-170); scale =
 * 2 * p_scale * sqrt(nx*ny*nz).  y: complex64 device array, out: float32. */
int mm_gp_finish(const void* y, int nx, int ny, int nz, float scale, float first, float last, float* out,
                 void* stream);

/* Vessel occupancy (optics.py:171-196): raw[x,y,c] = occ + raw[x,y,c] *
 * (1 - occ/denom), occ = sum of vessels[x0+x, y0+y, z] over zbounds[c] <=
 * z < zbounds[c+1].  vessels: (vx,vy,vz) float32 device array; zbounds: HOST
 * array of nz+1 rising entries in 0..vz (nz <= 512). */
int mm_vessel_combine(const float* vessels, int vx, int vy, int vz, int x0, int y0, const int* zbounds,
                      float denom, float* raw, int nx, int ny, int nz, void* stream);

/* ------------------------------------------------------------------------
 * Local-PSF overlap-add render (RANA compact-support operator), FP64.
 * One call renders the volume through one FullFieldPSF, or through every
 * field of a depth bank weighted per plane:
 *   out[r] += sum over fields f and node pairs (i,j) of the pair's tile
 *             correlation / convolution, weighted as the reference weights it.
 * Replaces LocalFFTPlan.__call__, maomi/rana/_fft.py:74-95 (with the plan
 * construction of :9-49 done on the host by mm_local_tiles), and the
 * per-field loop of RanaOperator.static, maomi/rana/operator.py:122-134.
 */
typedef struct {
  int sx, sy, sz;          /* volume shape (X,Y,Z)                              */
  int kx, ky, kz;          /* kernel shape                                      */
  int nodes_x, nodes_y;    /* field nodes                                       */
  const double* kernels;   /* (nfields, nodes_x, nodes_y, kx, ky, kz)           */
  const double* wx;        /* (nodes_x, sx) lateral weights                     */
  const double* wy;        /* (nodes_y, sy)                                     */
  int detection;           /* 1: weight sources before convolving              */
  int correlate;           /* 1: flipped kernel (excitation)                   */
  int plane;               /* 1: 2-D per-plane, output summed over z (scan_slab) */
  int nfields;             /* depth fields in `kernels` (1 unless a bank)       */
  const int32_t* tiles_x;  /* excitation/native: device copy of mm_local_tiles  */
  int ntiles_x;            /*   of wx (ignored for detection)                   */
  const int32_t* tiles_y;  /*   and of wy                                       */
  int ntiles_y;
} mm_local_desc;

/* Host-side plan step (no device work): split the output pixels [0, n) of one
 * axis into tiles over which the set of nodes with nonzero weight in
 * w (nodes, n; HOST array) is constant and at most 4 nodes, each at most
 * max_len (<= 18; 0 = 18) pixels long.  Writes up to `capacity` records of 8
 * int32 {start, length, active count, node[4], 0} to `table` (may be NULL)
 * and returns the number of tiles (n is always enough capacity), or a
 * negative status.  Counterpart of the node-pair tiling of
 * maomi/rana/_fft.py:24-49. */
int mm_local_tiles(const double* w, int nodes, int n, int max_len, int32_t* table, int capacity);

/* Bytes of device workspace mm_local_render needs (the source transposed). */
size_t mm_local_render_workspace_size(const mm_local_desc* desc);

/* zweight: (nfields, sz) device array or NULL (nfields == 1, weight 1):
 * excitation/native weight output plane z, detection weights source plane z.
 * Plane mode takes one field and no zweight (weight the source beforehand).
 * `out` is accumulated into. */
int mm_local_render(const mm_local_desc* desc, const double* source /* (sx,sy,sz) */,
                    const double* zweight, double* out /* (sx,sy[,sz]) */,
                    void* workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------------
 * BF16 tensor-core GEMM (tcgen05, FP32 accumulation), the building block of
 * the surrogate's spectral and pointwise layers:
 *   d[m x n] (FP32, row-major) = a[m x k] * b[n x k]^T   (a, b BF16, row-major)
 * n and k multiples of 16; a and b 16-byte aligned.  `err` is a zeroed device
 * int that a timed-out pipeline wait sets.  No reference counterpart: the
 * reference's surrogate-free stage has no GEMM; this is the kernel the
 * planned mm_surrogate_* entry points are built on, exported for testing.
 */
int mm_gemm_bf16_tn(const void* a, const void* b, float* d, int m, int n, int k, int* err, int check,
                    void* stream);

/* ------------------------------------------------------------------------
 * Learned PSF surrogate (Fourier neural operator, 4 layers of width 32,
 * 12 x 12 retained modes, BF16 tensor-core GEMMs with FP32 accumulation).
 * No reference counterpart: the reference has no learned component.  A
 * site's input is its 64 x 64 window of 16 pooled screen groups (plus two
 * coordinate channels); its output the 64 x 64 x 9 focal PSF, unit sum.
 * All buffers are device memory the caller allocates; BF16 matrices are
 * row-major.  Shapes for S sites:
 *   constants  F (576,4096), G (4096,576), FT = F^T, GT = G^T
 *   params     FP32 flat vector, layout from mm_surrogate_layout; grads same
 *   wb[l]/wtb[l] (32,32) BF16 copies of W_l and W_l^T; wlb (32,32); wpb (16,32); wptb (32,16)
 *   base (4096,16) FP32 mean PSF added to the projection
 *   xp (S*4096,32) / xc (S*32,4096) inputs; hp[l]/hc[l] (l = 0..4) activations, same shapes
 *   z[l] (S,4096,32) FP32 pre-activations (l = 0..2 needed for backward)
 *   v[l] (S,576,32) FP32 spectral coefficients (written only when z[0] is
 *   set: the mixing backward reads them); voc (S*32,576) BF16 scratch
 *   y (S,4096,16) FP32 prediction (planes 0..8 used)
 *   backward: dyp (S*4096,16), dyc (S*16,4096), dzp[2] (S*4096,32), dzc[2]
 *   (S*32,4096) BF16; dvo (S,576,32) FP32; dvc (S*32,576) BF16
 *   err: zeroed device int (bit 1: site off the input grid, bit 4: a
 *   tensor-core pipeline wait timed out)
 *   vb (288,S,64) BF16 spectral coefficients mode-major (row (q, s): the
 *   re and im rows of mode q, 32 channels each), the tensor-core mixing's A
 *   mixb[l] (288*64,64) BF16 per-mode mixing operators (filled from Rr/Ri by
 *   the forward pass; row 64 q + 2 o + c, c = 0 real / 1 imaginary output)
 */
typedef struct {
  int sites;
  const void* F;
  const void* G;
  const void* FT;
  const void* GT;
  float* params;
  float* grads;
  void* wb[4];
  void* wtb[4];
  void* wlb;
  void* wpb;
  void* wptb;
  const float* base;
  const void* xp;
  const void* xc;
  void* hp[5];
  void* hc[5];
  float* z[4];
  float* v[4];
  void* voc;
  float* y;
  void* dyp;
  void* dyc;
  void* dzp[2];
  void* dzc[2];
  float* dvo;
  void* dvc;
  int* err;
  void* vb;
  void* mixb[4];
} mm_surrogate_desc;

/* Offsets (floats) of Wl, bl, {W_l, b_l, Rr_l, Ri_l} for l = 0..3, Wp, bp and the total (21 entries). */
int mm_surrogate_layout(long long* offsets, int n);
/* Fill the BF16 spectral matrices. */
int mm_surrogate_constants(void* F, void* G, void* FT, void* GT, void* stream);
/* Prediction y for d->sites sites (refreshes the BF16 weight copies first). */
int mm_surrogate_forward(const mm_surrogate_desc* d, int check, void* stream);
/* Inference: the forward pass with the projection writing the PSF planes
 * planes (S,9,64,64) FP32, negatives clipped to 0, instead of y (the
 * equivalent of mm_surrogate_forward followed by mm_surrogate_planes). */
int mm_surrogate_predict(const mm_surrogate_desc* d, float* planes, int check, void* stream);
/* Loss (mean over sites of ||y - t||^2 / ||t||^2, planes 0..8) and every
 * parameter gradient into d->grads, after mm_surrogate_forward on the same d.
 * target: (S,4096,16) FP32. */
int mm_surrogate_backward(const mm_surrogate_desc* d, const float* target, double* loss, int check, void* stream);
/* One Adam step (bias-corrected, step >= 1) over n parameters. */
int mm_surrogate_adam(float* params, const float* grads, float* m, float* v, long long n, float lr, float beta1,
                      float beta2, float eps, int step, void* stream);
/* Site inputs from the raw A/B/C fields (each (h, w, z_part) FP32): screens
 * grouped by groups[0..16] (global screen index ranges), 4x4-pooled into
 * pooled (16, h/4, w/4), times scale; then each site's 64 x 64 window at
 * offsets/4 (offsets multiples of 4) into xp / xc. */
int mm_surrogate_inputs(const float* const* raw, const int* zpart, int h, int w, const int* groups, float scale,
                        float* pooled, const int* offsets, int sites, void* xp, void* xc, int* err, int check,
                        void* stream);
/* y (S,4096,16) -> PSF planes (S,9,64,64), negatives clipped to 0. */
int mm_surrogate_planes(const float* y, float* out, int sites, void* stream);

/* ------------------------------------------------------------------------
 * Static and per-frame scan operators: 2-D linear convolutions of real
 * planes with real kernel planes through zero-padded 2-D DFTs (sizes
 * fx x fy: 64, 128, 256, 512, 1024, and for FP32 planes 384 and 768) and a
 * per-bin coupling rule along Z.
 *
 * Replaces:
 *   zstack                 maomi/scanning.py:8-53   (CONV_Z / CORR_Z rules)
 *   psf_fft, _group_z      maomi/movie.py:32-42     (mm_scan_kernel_spectrum)
 *   single_scan            maomi/movie.py:48-66     (SUM_Z rule)
 *   blurred_background     maomi/movie.py:69-102    (mm_scan_background + EACH_Z)
 *   conv2_same             maomi/movie.py:14-19     (EACH_Z, one plane)
 *
 * Data are float32 (fp64 = 0, FP32 transforms) or float64 (fp64 = 1, FP64
 * transforms).  Planes are addressed through element strides, so slabs of a
 * larger (X, Y, Z) array need no copy.  Transform planes are packed two to
 * a complex transform; spectra stay on the device.
 * ------------------------------------------------------------------------ */
enum {
  MM_SCAN_CONV_Z = 0, /* out[o] = sum_l src[o + zoff - l] * k[l]  (3-D convolution, zero extended)   */
  MM_SCAN_CORR_Z = 1, /* out[o] = sum_l src[o - zoff + l] * k[l]  (correlation along Z, zero extended) */
  MM_SCAN_SUM_Z = 2,  /* out[0] = sum_z src[z] * k[z]              (one frame: sum of plane convolutions) */
  MM_SCAN_EACH_Z = 3  /* out[z] = src[z] * k[z]                    (independent planes) */
};

typedef struct {
  const void* data;       /* element (x, y, z) at data[x*s0 + y*s1 + z*s2] */
  long long s0, s1, s2;   /* element strides */
  int nx, ny, nz;         /* extents */
  int group;              /* consecutive planes summed into one transform plane (scan_avg); >= 1 */
  const void* mask0;      /* optional nx*ny row-major multipliers of every plane (NULL: none) */
  const void* mask1;
  const void* data2;      /* optional second volume of the same layout, added element-wise (NULL: none) */
} mm_scan_planes;

typedef struct {
  int fp64;               /* 0: float32 data / FP32 transforms; 1: float64 / FP64 */
  int fx, fy;             /* transform sizes: 64, 128, 256, 512, 1024; 384, 768 with fp64 = 0 */
  int kx, ky;             /* kernel plane extents */
  int kplanes;            /* kernel transform planes (after grouping) */
} mm_scan_desc;

typedef struct {
  mm_scan_planes src;
  int wrap;               /* 1: periodic extension: transform input row i = source row (i + wrap_x0) mod nx */
  int wrap_x0, wrap_y0;
  int ext_x, ext_y;       /* nonzero transform-input rows / columns (nx, ny without wrap) */
  int zrule;              /* MM_SCAN_* */
  int zoff;               /* Z offset of the CONV / CORR rules (kernel planes / 2) */
  int out_planes;         /* output planes (1 for SUM_Z) */
  int crop_x, crop_y;     /* first kept row / column of the linear convolution */
  int out_x, out_y;       /* kept rows / columns */
  void* out;              /* element (x, y, o) at out[x*o0 + y*o1 + o*o2], data type of the call */
  long long o0, o1, o2;
  int accumulate;         /* 1: out += alpha * result; 0: out = alpha * result */
  double alpha;
  const void* src_spectra;  /* non-NULL: packed source spectra (ceil(planes/2), fx, fy) from mm_scan_forward;
                               the forward pass is skipped and the spectra are left unchanged */
  void* out_spectra;        /* non-NULL: stop after the Z rule and store (accumulate 0) or add (1) the packed
                               output spectra (ceil(out_planes/2), fx, fy) there; `out` is not used */
  const void* out_weight;   /* non-NULL: (out_x, out_y) row-major weights of the kept window, times alpha */
} mm_scan_conv;

/* Bytes of a kernel spectrum (kplanes half spectra fx x (fy/2+1), complex). */
size_t mm_scan_spectrum_bytes(const mm_scan_desc* desc);
/* Bytes of workspace for `planes` transform planes (packed complex spectra). */
size_t mm_scan_workspace_size(const mm_scan_desc* desc, int planes);
/* Spectra of the (grouped) kernel planes into `spectrum` (psf_fft). */
int mm_scan_kernel_spectrum(const mm_scan_desc* desc, const mm_scan_planes* kernel, void* spectrum,
                            void* workspace, size_t workspace_bytes, void* stream);
/* One convolution pass: forward DFT of the (grouped, masked, optionally
 * wrapped) source planes, the Z rule against `spectrum`, inverse DFT, crop,
 * scale and store or accumulate. */
int mm_scan_convolve(const mm_scan_desc* desc, const mm_scan_conv* conv, const void* spectrum, void* workspace,
                     size_t workspace_bytes, void* stream);
/* Packed spectra (ceil(planes/2), fx, fy) of conv->src (grouping, masks,
 * wrap as in mm_scan_convolve): a source transformed once and reused by
 * several mm_scan_convolve calls through conv->src_spectra.  Replaces the
 * shared source spectrum of CubicFullFieldRenderer.__call__,
 * maomi/rana/fields.py:248-256. */
int mm_scan_forward(const mm_scan_desc* desc, const mm_scan_conv* conv, void* spectra, void* stream);
/* The inverse passes alone: packed spectra (ceil(conv->out_planes/2), fx, fy),
 * overwritten, to conv->out with its crop, weights, alpha and accumulate
 * (the final inverse of an accumulated spectrum, maomi/rana/fields.py:265). */
int mm_scan_inverse(const mm_scan_desc* desc, const mm_scan_conv* conv, void* spectra, void* stream);
/* The background source plane of blurred_background (movie.py:86-95):
 * out[x,y] = power * mask[x,y] / n * sum_i scale[i] * sum_v vol_v[x,y,idx[i]]
 * over nvol volumes that share one layout (s0, s1, s2); mask may be NULL.
 * idx: (n) int32 device array; scale: (n) float64 device array. */
int mm_scan_background(int fp64, const void* const* volumes, int nvol, long long s0, long long s1, long long s2,
                       int nx, int ny, int nz, const int32_t* idx, const double* scale, int n, double power,
                       const void* mask, void* out, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* MAOMI_B200_H */
