/*
 * pyspectral_b200 -- C ABI of the B200-native PySpectral right-hand-side and
 * RK4 path.
 *
 * Plain pointers and sizes only.  Every field argument is a DEVICE pointer to
 * a dense array of `nfields` spectra laid out (nfields, N1, N2, N3/2+1),
 * complex interleaved (re, im), FP64 or FP32 according to the context's
 * precision.  All work is queued on the context's stream; functions that
 * return host scalars synchronise that stream.  Every entry point returns a
 * status code (PSB_OK on success) and never aborts; psb_last_error() gives
 * the message.  A context is not thread-safe: use one per host thread/stream.
 *
 * Paths in citations are relative to the PySpectral project.
 */
#ifndef PYSPECTRAL_B200_H
#define PYSPECTRAL_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define PSB_OK 0
#define PSB_ERR_ARG 1         /* null pointer / bad value */
#define PSB_ERR_SHAPE 2       /* unsupported grid size */
#define PSB_ERR_CUDA 3        /* a CUDA call failed */
#define PSB_ERR_UNSUPPORTED 4 /* closure/precision combination not built */
#define PSB_ERR_NONFINITE 6   /* NaN/Inf detected by psb_check_finite */

/* ---- closures: the reference's turb_model switch
 *      (src/Classes.py:28-229, src_MPI/Classes.py:59-149) ----------------- */
#define PSB_DNS 0         /* turb_model 0      -> computeRHS_NOSGS  (src/RHSfunctions.py:3-50)    */
#define PSB_SMAG 1        /* turb_model 1      -> computeRHS_SMAG   (src/RHSfunctions.py:146-237)  */
#define PSB_TMODEL 2      /* turb_model 2      -> computeRHS_tmodel (src/RHSfunctions.py:240-363)  */
#define PSB_TAU_STATIC 3  /* 'Static tau-model'  (src/RHSfunctions.py:366-497)                       */
#define PSB_TAU_DYNAMIC 4 /* 'Dynamic tau-model' (src/RHSfunctions.py:592-878)                       */
#define PSB_MHD 5         /* 'MHD' of the MPI solver (src_MPI/RHSfunctions.py:95-175)                */
#define PSB_LEARNED 6     /* learned MLP subgrid stress (no reference counterpart; replaces the
                             Smagorinsky stress of src/RHSfunctions.py:195-212)                    */
#define PSB_MHD_TMODEL 7  /* MHD + t-model memory term Ct t PLQL on both fields (no reference
                             counterpart; the construction of src/RHSfunctions.py:240-363 applied
                             to src_MPI/RHSfunctions.py:95-175, resolved set = 2/3-rule set)      */
#define PSB_DSMAG 8       /* turb_model 7      -> computeRHS_DSMAG  (src/RHSfunctions.py:1663-1862):
                             Smagorinsky with Cs^2 = <L:M>/<M:M> from the test filter
                             myFilter(., kc/2) (src/Classes.py:1271-1279)                          */
#define PSB_CM1 9         /* turb_model 6      -> computeRHS_CM1    (src/RHSfunctions.py:1411-1542):
                             6 fields u,v,w,w0_u,w0_v,w0_w; du/dt = unpad_2x(PLu) + w0,
                             dw0/dt = PLQLu - 250 nu k^2 w0; w0_v read as zero like the
                             reference's Q2U (src/Classes.py:489); no rotating form           */
#define PSB_FM1 11        /* turb_model 3      -> computeRHS_FM1    (src/RHSfunctions.py:882-1024):
                             3 + 3 p.fm_nsub fields u, then (w0_u, w0_v, w0_w) per
                             subintegration; du/dt = unpad_2x(PLu) + sum_i w0_i,
                             dw0_i/dt = -2/d w0_i + (-1)^(i+1) 2 PLQLu + S_i, d = dt0/nsub,
                             S_i the running sum of :1010-1014; w0 (3 p.fm_nsub fields)
                             receives the memory variables as read                          */
#define PSB_FM2 15        /* turb_model 4      -> computeRHS_FM2    (src/RHSfunctions.py:1025-1286):
                             3 + 6 p.fm_nsub fields u, then per subintegration i the
                             pairs w0^i (fields 3+6i..) and w1^i (fields 6+6i..), the
                             interleaved layout of src/Classes.py:330-355 with equal
                             dt0/dt1 subintegrations; du/dt = unpad_2x(PLu) + sum_i w0^i,
                             dw0^i/dt = -2/d0 w0^i + (-1)^(i+1) 2 PLQLu + S0_i + w1^i,
                             dw1^i/dt = -2/d1 w1^i + (-1)^(i+1) 2 PLQLQLu + S1_i
                             (d0 = fm_dt0/nsub, d1 = fm_dt1/nsub); PL x PL_q products on
                             the 3N grid; w0 (6 p.fm_nsub fields, w0^i then w1^i per i)
                             receives the memory variables as read; no rotating form      */
#define PSB_ORTHO 12      /* 'Orthogonal Dynamics' -> computeRHS_Orthogonal (src/RHSfunctions.py:53-143):
                             the DNS RHS of u minus the DNS RHS of Gf u (each with its
                             pressure and Coriolis terms)                                     */
#define PSB_MPI_DNS 13    /* MPI solver turb_model 0 -> computeRHS_NOSGS (src_MPI/RHSfunctions.py:22-93):
                             2/3-rule dealiasing on the N grid (no padding), + rotation           */
#define PSB_MPI_ORTHO 14  /* MPI solver 'Orthogonal Dynamics' -> computeRHS_Ortho
                             (src_MPI/RHSfunctions.py:179-268): the PSB_MPI_DNS RHS of u minus
                             that of grid.filter(u) (cutoff kc, src_MPI/Classes.py:219-235)   */
#define PSB_BUDGETS 10    /* turb_model 99     -> computeRHS_BUDGETS (src/RHSfunctions.py:1543-1661):
                             RHS = unpad_2x(PLu); w0 receives PLQLu with the q part split at
                             p.kf (0 -> int(max k1), main.kc of src/Classes.py:16); no
                             rotating form                                                      */

/* ---- diagnostic flags --------------------------------------------------- */
#define PSB_NORM_SERIAL 0   /* divide by N1*N2*N3      (src/Classes.py:652-659)      */
#define PSB_NORM_MPI 1      /* divide by (N1*N2*N3)^2  (src_MPI/Classes.py:269-285)  */
#define PSB_FILTER_GF 2     /* apply the sharp cutoff Gf first (src/Classes.py:584-588) */
#define PSB_TRANSFER_2D 4   /* psb_transfer / psb_spectrum_nbins: the *_2D transfer variants
                               (src/Classes.py:1043-1092,1152-1205,1241-1270) */

typedef struct psb_ctx psb_ctx;

/* gridclass(N1,N2,N3,x,y,z,kc,L1,L2,L3) (src/Classes.py:548-588).  dx,dy,dz
 * are the spacings of the caller's coordinate arrays (Delta=(dx dy dz)^(1/3)). */
typedef struct {
  int N1, N2, N3;
  double L1, L2, L3;
  double dx, dy, dz;
  int kc;
} psb_grid;

/* Run parameters carried by the reference's `variables` object
 * (src/Classes.py:8-26, defaults src/PySpec_3d.py:9-72). */
typedef struct {
  double nu;           /* viscosity */
  double eta;          /* magnetic diffusivity; <0 -> nu (src_MPI/Classes.py:95) */
  double t;            /* time, frozen across the four stages (src/PySpec_3d.py:122) */
  double dt;           /* time step */
  double Ct;           /* t-model constant (src/Classes.py:103-108) */
  double tau_a, tau_b; /* static tau-model tau = max(0, tau_a + tau_b t) (src/Classes.py:194-195) */
  int kf;              /* dynamic tau test-filter wavenumber; 0 -> int(kc*2/3) (src/Classes.py:131);
                          PSB_BUDGETS: the budget split main.kc; 0 -> int(max k1) (src/Classes.py:16) */
  int rotate;          /* Coriolis on/off (src/RHSfunctions.py:33-36,47-50) */
  double Om1, Om2, Om3;
  const void* force;   /* MHD: constant forcing spectra, 3 fields, or NULL (src_MPI/Classes.py:91-94) */
  const void* mlp_params; /* PSB_LEARNED: FP32 parameter block (psb_mlp_sizes) on the device */
  const void* mlp_norm;   /* PSB_LEARNED: FP32 normalisation block on the device */
  double les_delta;       /* PSB_LEARNED: filter width fed to the MLP; <=0 -> (dx dy dz)^(1/3) */
  int mlp_act;            /* PSB_LEARNED: hidden activation of the model, PSB_ACT_GELU or PSB_ACT_RELU */
  int mlp_hidden;         /* PSB_LEARNED: hidden width of the model, 32 or 64 (0 = 64) */
  double fm_dt0;          /* PSB_FM1: memory length dt0 (src/Classes.py:236-241; default 0.1) */
  int fm_nsub;            /* PSB_FM1: dt0_subintegrations, 1..8 (0 = 1) (src/Classes.py:243-248);
                             PSB_FM2: dt0_ and dt1_subintegrations (equal), 1..8 */
  double fm_dt1;          /* PSB_FM2: second memory length dt1 (src/Classes.py:302-308; default 0.05) */
} psb_params;

/* Hidden activation of the learned closure's MLP (a property of the trained model). */
#define PSB_ACT_GELU 0 /* x Phi(x) */
#define PSB_ACT_RELU 1 /* max(x, 0) */

/* FFTclass + gridclass construction (src/Classes.py:548-625; src/PySpec_3d.py:79-80).
 * precision: 32 or 64.  N1,N2,N3 must be multiples of 4 whose 3/2 and 2x
 * padded sizes factor as 2^a 3^b (8,12,16,24,32,48,64,96,128,192,256,...). */
int psb_ctx_create(const psb_grid* grid, int precision, int device, psb_ctx** out);
int psb_ctx_destroy(psb_ctx* ctx);
/* Stream (cudaStream_t) on which the context queues its work; NULL = legacy default. */
int psb_ctx_set_stream(psb_ctx* ctx, void* stream);
/* Stage the inputs of the passes that read their rows unchanged (forward y
 * pass, the x pass of the spectral epilogue, plain inverse y passes) with
 * bulk tensor copies (1, the default) or with per-element loads (0).  Same
 * results either way; no counterpart in the reference (a launch choice). */
int psb_ctx_set_tma(psb_ctx* ctx, int enable);
/* Run the z pass of the 3/2-padded Navier-Stokes closures (DNS products,
 * Smagorinsky, learned; FP32) with its spectra loaded into and stored from
 * registers around the transforms when its schedule is a compiled two-pass
 * one ending in radix 16 (1, the default), or through shared memory (0).
 * Same results either way; no counterpart in the reference (a launch choice). */
int psb_ctx_set_zrr(psb_ctx* ctx, int enable);
/* Device status of the context's kernels since the last call, then cleared:
 * 0; 1 when a bounded wait inside a kernel gave up; 2 when a kernel found a
 * bulk-copy destination off its alignment and issued nothing.  In both cases
 * that kernel wrote NaN in place of the tile it could not stage instead of
 * hanging or faulting.  Synchronises the context stream.  No counterpart in
 * the reference (it has no device). */
int psb_device_status(psb_ctx* ctx, int* status);
/* Message of the last failure on this context ("" if none). */
const char* psb_last_error(const psb_ctx* ctx);
/* Message of the last psb_ctx_create failure (no context exists then). */
const char* psb_create_error(void);

/* One right-hand-side evaluation: main.computeRHS(main,grid,myFFT,utilities)
 * (src/Classes.py:44,95,124,186,227; src_MPI/Classes.py:147).
 * state (read) and rhs (written) hold 3 fields (6 for PSB_MHD, PSB_MHD_TMODEL, PSB_CM1;
 * 3 + 6 p.fm_nsub for PSB_FM2;
 * 3 + 3 p.fm_nsub for PSB_FM1).
 * w0       : optional closure force main.w0_u/v/w (3 fields; 6 fields u then B for
 *            PSB_MHD_TMODEL) or NULL.
 * read_out : optional copy of the state as the RHS read it (the reference
 *            rebinds main.uhat/vhat/what to it, src/RHSfunctions.py:10-12;
 *            the MPI solver dealiases it in place, src_MPI/RHSfunctions.py:102-107).
 * tau_out  : optional host scalar main.tau (tau-models; src/RHSfunctions.py:480,857);
 *            for PSB_DSMAG the dynamic coefficient Cs_sqr (:1843). */
int psb_rhs(psb_ctx* ctx, int closure, const void* state, void* rhs, void* w0, void* read_out,
            const psb_params* p, double* tau_out);

/* DNS right-hand side (same result as psb_rhs with PSB_DNS) that allocates no
 * device memory.  No counterpart in the reference.  For callers that cannot
 * call cudaMalloc when they evaluate the RHS: hosts whose pool allocator owns
 * the device memory (a library cudaMalloc would fail), time-critical loops
 * that cannot take cudaMalloc's implicit synchronisation.  Scratch is a fixed
 * 8,847,360-byte __device__ array in the library; a grid needs
 * 16.875 * N1*N2*N3 complex elements of it (each buffer rounded up to 256 B),
 * so N1*N2*N3 may be at most 32^3 in FP64 and 2*32^3 in FP32 (e.g. 32^3 or
 * 32x32x64); larger grids return PSB_ERR_SHAPE.  The first call on a device
 * looks up the array's address (make it before any stream capture).  All
 * calls share the array, so calls that overlap on the GPU race; serialise
 * them.  The caller's current device is left as it was.  The context itself
 * must already exist (psb_ctx_create allocates). */
int psb_rhs_dns_noalloc(psb_ctx* ctx, const void* state, void* rhs, const psb_params* p);

/* nsteps of advanceQ_RK4 (src/PySpec_3d.py:96-105; src_MPI/time_schemes.py:2-7):
 * Q <- Q0 + dt*c_i*RHS(Q), c = [1/4,1/3,1/2,1], in place on `state`.
 * comp     : Kahan compensation array (same shape as state) for FP32 runs, or NULL.
 * read_out : optional; receives the state read by the LAST stage of the LAST
 *            step (the reference's per-step diagnostics read main.uhat,
 *            src/PySpec_3d.py:129).  dt is fixed (cfl<=0 in compute_dt).
 * For an unsupported graph-captured first call see psb_prepare. */
int psb_step_rk4(psb_ctx* ctx, int closure, void* state, void* comp, void* read_out, const psb_params* p,
                 int nsteps);

/* nsteps of the MPI solver's semi-implicit scheme for Navier-Stokes, advanceQ_SI
 * (src_MPI/time_schemes.py:9-11) with the 'Semi-Implicit' branch of computeRHS_NOSGS
 * (src_MPI/RHSfunctions.py:70-93), in place on `state` (3 fields):
 *   H <- the 2/3-masked nonlinear term (+ Coriolis),
 *   Q <- (Q + dt/2 (3 H - H_old) + dt/2 (-nu k^2 u)) / (1 + nu dt/2 k^2).
 * H (3 fields) holds H_old on entry and the last step's H on exit; start it at
 * zero (the reference allocates it with np.empty).  read_out: optional, the
 * masked state the last step read (main.uhat). */
int psb_step_si(psb_ctx* ctx, void* state, void* H, void* read_out, const psb_params* p, int nsteps);

/* Allocate the context's scratch for `closure` now (so that a later call can
 * be captured in a CUDA graph without allocating). */
int psb_prepare(psb_ctx* ctx, int closure);

/* ---- diagnostics (FP64 results on the host) ----------------------------- */
/* computeEnergy / computeEnergy_resolved (src/Classes.py:652-676), MPI
 * computeEnergy / computeMHDEnergy (src_MPI/Classes.py:269-303). 3 fields. */
int psb_energy(psb_ctx* ctx, const void* fields3, int flags, double* out);
/* computeEnstrophy (src/Classes.py:733-744; src_MPI/Classes.py:350-368). */
int psb_enstrophy(psb_ctx* ctx, const void* fields3, int flags, double* out);
/* Cross-helicity <u.B> with the MPI energy weighting (no reference counterpart). */
int psb_cross_helicity(psb_ctx* ctx, const void* u3, const void* b3, int flags, double* out);
/* computeSpectrum / computeSpectrum_resolved (src/Classes.py:762-797,825-844):
 * out[nbins*3] (row-major [bin][component]), int8 shell index with the
 * reference's wrap-around.  nbins must be the reference's kmax+1
 * (psb_spectrum_nbins). */
int psb_spectrum(psb_ctx* ctx, const void* fields3, int flags, double* out, int nbins);
int psb_spectrum_nbins(const psb_ctx* ctx, int flags, int* nbins);
/* computeTransfer (src/Classes.py:988-1040): energy transfer spectrum of the
 * 3 fields (Nyquist modes treated as zero, 3/2-dealiased products), binned
 * like psb_spectrum; out[2*nbins] = (Re, Im) per bin, nbins from
 * psb_spectrum_nbins(ctx, 0, &nbins).  flags PSB_FILTER_GF:
 * computeTransfer_resolved (:1093-1150, the fields filtered by Gf).  w0 (3
 * fields) non-NULL: computeTransfer_SGS (:1206-1239), Re sum_i conj(Gf u_i) w0_i.
 * flags PSB_TRANSFER_2D: the *_2D variants of the three (:1043-1092,
 * :1152-1205, :1241-1270): the k3 = 0 plane only, bins rint(sqrt(k1^2+k2^2)),
 * u and v only, weight 1; nbins from psb_spectrum_nbins(ctx, PSB_TRANSFER_2D, &nbins). */
int psb_transfer(psb_ctx* ctx, const void* fields3, const void* w0, int flags, double* out, int nbins);
/* MPI computeSpectrum / computeMHDSpectrum (src_MPI/Classes.py:370-448):
 * out[nbins] summed over components, int16 shells, k3=N/2 included. */
int psb_spectrum_mpi(psb_ctx* ctx, const void* fields3, double* out, int nbins);
/* compute_dt (src/Classes.py:687-698): CFL time step for cfl>0, else -cfl. */
int psb_cfl_dt(psb_ctx* ctx, const void* fields3, double cfl, double nu, double* dt_out);
/* computeSGS_DNS (src/Classes.py:861-929): w0 (3 fields) and optional tauhat (6 fields). */
int psb_sgs_dns(psb_ctx* ctx, const void* fields3, void* w0, void* tau6);

/* ---- transforms and setup ----------------------------------------------- */
/* numpy rfftn (unnormalised) of nfields physical fields (N1,N2,N3) real. */
int psb_fft_r2c(psb_ctx* ctx, const void* phys, void* spec, int nfields);
/* numpy irfftn (1/(N1N2N3)-normalised) of nfields spectra. */
int psb_fft_c2r(psb_ctx* ctx, const void* spec, void* phys, int nfields);
/* Slab-decomposed 3-D transforms of the MPI solver, FFTclass.myifft3D /
 * myfft3D (src_MPI/Classes.py:244-258), for one rank of nprocs.  The rank holds
 * the spectra of an x slab, (Npx, N2, Kz), and the physical field of a y slab,
 * (N1, Npy, N3), with Npx = N1/nprocs, Npy = N2/nprocs, Kz = N3/2+1 (N1 and N2
 * multiples of nprocs; ctx is a context of the whole N1 x N2 x N3 grid).
 * Between the two halves of each transform the caller runs an all-to-all of
 * nprocs equal blocks (block p of `send` to rank p, block p of `recv` from rank
 * p), as the reference's comm.Alltoall does; one field per call.
 *   psb_slab_ifft_y : uhat (Npx, N2, Kz) -> send (nprocs, Npx, Npy, Kz), the
 *                     inverse DFT along y, block p = rank p's y rows
 *   psb_slab_ifft_xz: recv (N1, Npy, Kz) -> u (N1, Npy, N3) real: inverse DFT
 *                     along x, c2r along z, scaled by 1/(N1 N2 N3) (numpy's ifft
 *                     and irfft2 normalisation together)
 *   psb_slab_fft_xz : u (N1, Npy, N3) -> send (N1, Npy, Kz): r2c along z, DFT
 *                     along x (unnormalised); block p = rank p's x rows
 *   psb_slab_fft_y  : recv (nprocs, Npx, Npy, Kz) -> uhat (Npx, N2, Kz): the DFT
 *                     along y (unnormalised) */
int psb_slab_ifft_y(psb_ctx* ctx, int nprocs, const void* uhat, void* send);
int psb_slab_ifft_xz(psb_ctx* ctx, int nprocs, const void* recv, void* u);
int psb_slab_fft_xz(psb_ctx* ctx, int nprocs, const void* u, void* send);
int psb_slab_fft_y(psb_ctx* ctx, int nprocs, const void* recv, void* uhat);
/* Count of non-finite values in n complex entries -> *count (0 = all finite). */
int psb_check_finite(psb_ctx* ctx, const void* data, long long n, long long* count);

/* ---- learned subgrid closure (no counterpart in the reference) ----------
 * MLP 10 -> H -> H -> 6 (hidden width H = hidden: 32 or 64, 0 meaning 64;
 * hidden activation act: PSB_ACT_GELU or PSB_ACT_RELU), BF16 tensor-core
 * math with FP32 accumulation.  Features: the 9 velocity gradients du_i/dx_j
 * (order 3i+j) and the filter width; targets: tau_11,22,33,12,13,23.
 * Parameters are an FP32 master block of *nparams floats (W1[H][10] b1[H]
 * W2[H][H] b2[H] W3[6][H] b3[6]), normalisation a block of *nnorm floats
 * (xmean[10] xistd[10] ymean[6] ystd[6]); all device pointers. */
int psb_mlp_sizes(int hidden, int* nparams, int* nnorm);
/* Y[B][6] = tau(X[B][10]) (raw units in and out). */
int psb_mlp_forward(psb_ctx* ctx, int act, int hidden, const float* params, const float* norm, const float* X, int B,
                    float* Y);
/* The same forward pass of a width-64 network on the fifth-generation tensor
 * cores (tcgen05.mma, 128-point tiles, FP32 accumulators in tensor memory).
 * err: optional device int set to 1 if an MMA did not complete within the
 * kernel's wait bound. */
int psb_mlp_forward_tc(psb_ctx* ctx, int act, const float* params, const float* norm, const float* X, int B, float* Y,
                       int* err);
/* grad += d(MSE of normalised outputs)/d(params) over the B points X[idx[b]],
 * T[idx[b]]; *loss (device double) += the MSE. */
int psb_mlp_grad(psb_ctx* ctx, int act, int hidden, const float* params, const float* norm, const float* X,
                 const float* T, const int* idx, int B, float* grad, double* loss);
/* One Adam(W) update of the width-`hidden` parameter block from grad (step >= 1); clears grad. */
int psb_mlp_adam(psb_ctx* ctx, int hidden, float* params, float* m, float* v, float* grad, int step, float lr,
                 float beta1, float beta2, float eps, float weight_decay);
/* Physical fields on the N grid (irfftn(uhat)*sqrt(N1N2N3)): what=0 -> u,v,w
 * (3 fields); what=1 -> u,v,w and the 9 gradients du_i/dx_j (12 fields). */
int psb_physical_fields(psb_ctx* ctx, const void* fields3, int what, void* out);
/* The six 3/2-dealiased product spectra u_i u_j (11,22,33,12,13,23) in the
 * state normalisation: uuhat... of src/RHSfunctions.py:18-23. */
int psb_products(psb_ctx* ctx, const void* fields3, void* out6);
/* Copy the modes |k_i| < kc (per axis, index units) of nfields spectra from a
 * (N1,N2,N3) grid to a (n1,n2,n3) grid times `scale`, all other modes zero
 * (sharp spectral cutoff and change of resolution).  precision 32 or 64;
 * stream is a cudaStream_t or NULL. */
int psb_spectral_resample(const void* src, int N1, int N2, int N3, void* dst, int n1, int n2, int n3, int nfields,
                          int kc, double scale, int precision, void* stream);

/* ---- launch accounting and per-kernel timing (no reference counterpart;
 *      the reference only prints wall time, src/PySpec_3d.py:107,136,144) --- */
/* Number of kernels this context has launched since creation. */
int psb_launch_count(const psb_ctx* ctx, unsigned long long* n);
/* Turn per-launch CUDA-event timing on/off; either call clears the records. */
int psb_timing_enable(psb_ctx* ctx, int on);
/* Synchronise the stream and return the number of timed launches. */
int psb_timing_count(psb_ctx* ctx, int* n);
/* Record i: kernel name, device time (ms) and compulsory HBM bytes of the launch. */
int psb_timing_get(psb_ctx* ctx, int i, char* name, int name_len, double* ms, double* bytes);

/* ---- batched ensembles (no reference counterpart: the reference advances one
 *      run per process, src/PySpec_3d.py:96-144) ------------------------------
 * nruns independent runs on ctx's grid and precision with one closure (PSB_DNS,
 * PSB_SMAG or PSB_LEARNED), each with its own state, Kahan compensation and
 * parameters (nu, dt, rotation, MLP).  Every pass of an RK4 stage is one launch
 * over all runs.  The batch owns its scratch; states stay caller-owned.  Calls
 * go to ctx's stream and may be captured into a CUDA graph once the batch has
 * stepped (or been tuned) outside the capture. */
typedef struct psb_batch psb_batch;
int psb_batch_create(psb_ctx* ctx, int closure, int nruns, psb_batch** out);
/* Run r: state (3 fields), comp (Kahan compensation, 3 fields, or NULL), params. */
int psb_batch_set_run(psb_batch* b, int r, void* state, void* comp, const psb_params* p);
/* Time the candidate launch shapes (column tiles, pencils per CTA, radix
 * orders) of every pass on the batch's data and keep the fastest; states are
 * not modified. */
int psb_batch_autotune(psb_batch* b);
/* nsteps RK4 steps of every run (src/PySpec_3d.py:96-105 per run). */
int psb_batch_step_rk4(psb_batch* b, int nsteps);
/* Launch shape of pass 0..4 (x-inverse, y-inverse, z, y-forward, x-forward):
 * tile (columns per CTA, or pencils per CTA for the z pass) and the radix
 * order of its transform (maxr entries, 0-terminated). */
int psb_batch_shape(const psb_batch* b, int pass, int* tile, int* radices, int maxr);
int psb_batch_destroy(psb_batch* b);

/* ---- persistent ensembles (no reference counterpart) ----------------------
 * Up to 4 batches on one device and precision (grid sizes and closures may
 * differ: PSB_DNS, PSB_SMAG, PSB_LEARNED with a ReLU width-32 network)
 * advanced together by ONE cooperative launch per call: the kernel walks the
 * RK4 stages and the five passes, spreading each pass's tiles over every run
 * of every batch, with a grid barrier between passes.  Every barrier wait is
 * bounded (poll_limit polls; 0 = the default of 2^26): a wait that gives up
 * raises the ensemble's status word and the kernel returns early (the states
 * are then partly advanced).  The batches' runs and shapes are read at each
 * call; step once outside a stream capture before capturing calls. */
typedef struct psb_ensemble psb_ensemble;
int psb_ensemble_create(psb_batch* const* batches, int nbatch, psb_ensemble** out);
int psb_ensemble_step_rk4(psb_ensemble* e, int nsteps, unsigned poll_limit);
/* 0, or 1 when a grid-barrier wait gave up since the last call (then cleared;
 * synchronises the first batch's stream). */
int psb_ensemble_status(psb_ensemble* e, int* status);
int psb_ensemble_destroy(psb_ensemble* e);

/* ---- autotuned single runs (no reference counterpart) --------------------
 * Time the candidate launch shapes of the five passes of closure's RHS
 * (PSB_DNS, PSB_SMAG or PSB_LEARNED) on `state` (not modified) with params p,
 * and keep the fastest in ctx: later psb_rhs / psb_step_rk4 calls of that
 * closure use them.  Results differ from the untuned ones only by rounding
 * (other radix orders). */
int psb_autotune(psb_ctx* ctx, int closure, void* state, const psb_params* p);
/* The tuned shape of pass 0..4 of closure (tile 0 when not tuned). */
int psb_tuned_shape(const psb_ctx* ctx, int closure, int pass, int* tile, int* radices, int maxr);
/* Back to the default shapes for closure. */
int psb_autotune_clear(psb_ctx* ctx, int closure);
/* Set the launch shape of pass 0..4 of closure (DNS, SMAG, LEARNED) by hand:
 * tile (columns per CTA, a power of two <= 32; pencils per CTA for the z pass,
 * a power of two <= the closure's bound) and the radix order of its transform
 * (nrad radices from {2,3,4,6,8,12,16} whose product is the pass's padded
 * length).  Replays a saved psb_autotune result (the pyFFTW plans of
 * src/Classes.py:590-625 carry no such choice: this is the autotuner's cache).
 * The other passes keep their tuned or default shapes. */
int psb_set_tuned_shape(psb_ctx* ctx, int closure, int pass, int tile, const int* radices, int nrad);

#ifdef __cplusplus
}
#endif
#endif /* PYSPECTRAL_B200_H */
