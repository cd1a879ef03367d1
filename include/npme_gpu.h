/*
 * npme_b200 — B200-native (sm_100a) potential evaluation for the
 * non-periodic particle-mesh Ewald method (NPME).
 *
 * C ABI.  Plain pointers and sizes, no C++ or torch types.  Every entry point
 * returns an npme_status and never exits the process; the message of the
 * last failure is available from npme_gpu_last_error().
 *
 * The calls replace the reference's interface classes (ElkingD/npme,
 * src/Interface.h) entry by entry:
 *
 *   reference                                          this ABI
 *   -------------------------------------------------  ---------------------------
 *   NPME_Interface_SetUpRealKernel / ComplexKernel     npme_gpu_create +
 *     (src/Interface.cpp:884, 1066), SetUp                npme_gpu_setup
 *     (src/Interface.h:393-395, 733-735)
 *   NPME_InterfaceReal::ResetCoord (src/Interface.h:188)  npme_gpu_setup
 *   NPME_InterfaceReal::CalcV      (src/Interface.h:192)  npme_gpu_calcv_real
 *   NPME_InterfaceComplex::CalcV   (src/Interface.h:525)  npme_gpu_calcv_complex
 *   NPME_InterfaceReal::CalcV_exact (src/Interface.h:200) npme_gpu_calcv_exact_real
 *   NPME_InterfaceComplex::CalcV_exact (src/Interface.h:532)
 *                                                      npme_gpu_calcv_exact_complex
 *   NPME_InterfaceReal::Print      (src/Interface.h:209)  npme_gpu_get_info
 *   NPME_KeywordInput defaults (src/Interface.cpp:53-517) npme_gpu_default_params
 *   (destructor)                                       npme_gpu_destroy
 *
 * Data layout is the reference's: coord[3n] xyz interleaved (double);
 * real charge[n] (double) or complex charge[2n] (re, im); output
 * V[n][4] = (V, dV/dx, dV/dy, dV/dz) as double, or as complex
 * (re, im) pairs, i.e. 8 doubles per point.  Outputs are in the caller's
 * particle order.  Unlike the reference, inputs are never modified.
 *
 * Semantics kept from the reference: CalcV assumes the coordinates given to
 * setup (geometry fixed, charges vary per call); setup again to change the
 * geometry.  CalcV = direct sum - f_LR(0) q + reciprocal sum; CalcV_exact is
 * the plain O(N^2) sum with no self term.
 */
#ifndef NPME_GPU_H
#define NPME_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  NPME_OK = 0,
  NPME_EINVAL = 1,   /* bad argument or parameter combination */
  NPME_ENOMEM = 2,   /* device or host allocation failed */
  NPME_ECUDA = 3,    /* CUDA / cuFFT error */
  NPME_ETIMEOUT = 4, /* a bounded device wait ran out */
  NPME_EBUSY = 5,    /* queue full */
  NPME_ESTATE = 6    /* call out of order (e.g. calcv before setup) */
} npme_status;

/* funcType keyword: "Laplace", "Ralpha", "Helmholtz"; NPME_FUNC_USER: a
 * caller-defined kernel (npme_gpu_set_user_kernel) */
enum { NPME_FUNC_LAPLACE = 0, NPME_FUNC_RALPHA = 1, NPME_FUNC_HELMHOLTZ = 2,
       NPME_FUNC_USER = 3 };
/* EwaldSplit keyword: "DerivMatch", "LaplaceOrig" */
enum { NPME_SPLIT_DERIVMATCH = 0, NPME_SPLIT_LAPLACE_ORIG = 1 };
/* Arithmetic of the bulk work.  FP64: everything in double ("plain").
 * FP32: spreading, FFT, interpolation and pair arithmetic in float with
 * per-target accumulation and the output in double. */
enum { NPME_PREC_FP64 = 0, NPME_PREC_FP32 = 1 };

/* Keyword-compatible parameters (names of the reference's keywords). */
typedef struct {
  int funcType;     /* NPME_FUNC_* */
  int EwaldSplit;   /* NPME_SPLIT_* */
  double alpha;     /* r^alpha exponent (Ralpha) */
  double k0_r;      /* Helmholtz wave number, real part */
  double k0_i;      /* Helmholtz wave number, imaginary part */
  double Rdir;      /* direct-space cutoff (required, > 0) */
  double tol;       /* original-Ewald tolerance (default 1e-6) */
  int nDeriv;       /* derivative-match order (default from BnOrder) */
  int BnOrder;      /* B-spline order, even, 4..16 (default 8) */
  long N1, N2, N3;  /* full FFT box, multiples of 4 (required) */
  long n1, n2, n3;  /* reference block size keywords; accepted, not used */
  double a1, a2, a3;       /* Fourier-extension window (default 4.0) */
  double del1, del2, del3; /* Fourier-extension margin (default Rdir) */
  int nNeigh;       /* direct-sum cells per Rdir (default 2) */
  int nCellClust1D; /* accepted for keyword compatibility, not used */
  int useCompactF;  /* accepted; both values give the same kernel */
  int precision;    /* NPME_PREC_* (default FP32) */
  int device;       /* CUDA device ordinal (default 0) */
} npme_params;

/* Read-back of the set-up state (the reference's Print). */
typedef struct {
  size_t nCharge;
  double X, Y, Z;       /* PME-corrected extents */
  double R[3];          /* translation used by the grid mapping */
  double L[3];          /* periodic lengths 2 (X + del) */
  double fself_r, fself_i; /* f_LR(0) */
  double dm_a_r[32], dm_a_i[32]; /* derivative-match coefficients a[n] */
  int nDeriv;
  long nCells, nBricks, nNonEmptyBricks;
  size_t deviceBytes;   /* device memory held by the handle */
  float stage_ms[8];    /* last calcv with timing on: gather, spread, fft,
                           multiply, ifft, direct, interp, total */
  int launches;         /* kernels launched by the last calcv */
  long nGroups;         /* direct sum: warp groups of <= 32 points */
  double candidatesPerPoint; /* direct sum: staged sources per target */
  int pairsOnce;        /* 1: the direct sum evaluates every pair once, for
                           both of its points (FP32 real DM kernels) */
  double pairsOnceCandidatesPerPoint; /* half-shell sources per target */
} npme_info;

typedef struct npme_handle npme_handle;

/* Fills the reference's defaults (src/Interface.cpp:53-517; src/Constant.h). */
void npme_gpu_default_params(npme_params *p);

/* Validates p and creates a handle on p->device.  No geometry yet. */
int npme_gpu_create(const npme_params *p, npme_handle **out);

/* Replaces the parameters of a handle (kernel, splitting, Rdir, B-spline
 * order, FFT box, precision ...; not the device).  Waits for the handle's
 * enqueued work, keeps its device buffers and takes its FFT plans from the
 * process-wide plan cache at the next setup, which must follow before CalcV.
 * No counterpart in the reference, whose interface objects are set up once;
 * it lets a server reuse one handle for requests with different
 * parameters.  On error the old parameters stay in force. */
int npme_gpu_set_params(npme_handle *h, const npme_params *p);

/* Caller-defined real kernels: the reference's generic interface
 * (NPME_InterfaceReal_GenFunc with NPME_KfuncReal functors for f, f_LR and
 * f_SR, src/Interface.h:302-304, src/KernelFunction.h:25-65).  On the GPU
 * the functors are device code: a caller writes a functor type in CUDA and
 * lets include/npme_user_kernel.cuh instantiate the three kernel-dependent
 * launches for it (direct sum, long-range sampling for the kernel
 * transform, exact sum); npme_user::ops<Functor>() returns this table.  The
 * handle must have funcType NPME_FUNC_USER; set the table before setup.
 * fself = f_LR(0), subtracted as the self term.  Real and complex kernels
 * (the reference's NPME_KfuncReal and NPME_KfuncComplex). */
typedef struct {
  double fself, fself_i;  /* f_LR(0) (imaginary part for complex kernels) */
  int complex_kernel;     /* 1: complex kernel (complex charges and V) */
  int (*direct)(npme_handle *h, const void *args, void *stream);
  int (*sample_lr)(npme_handle *h, int M1, int M2, int M3, const double *ax,
                   const double *ay, const double *az, void *out, void *stream);
  int (*exact)(npme_handle *h, const double *d_charge, double *d_V, void *stream,
               const unsigned int *d_targets, long n_targets);
} npme_user_ops;
int npme_gpu_set_user_kernel(npme_handle *h, const npme_user_ops *ops);

/* SetUp / ResetCoord: bins and sorts the points, builds the kernel transform,
 * the FFT plans and all work buffers.  coord is a host pointer. */
int npme_gpu_setup(npme_handle *h, size_t n, const double *coord);

/* CalcV with host buffers (real kernels).  coord may be NULL; when given it
 * must be the set-up geometry.  V: 4n doubles. */
int npme_gpu_calcv_real(npme_handle *h, double *V, size_t n,
                        const double *charge, const double *coord);

/* CalcV with host buffers (complex kernels).  charge: 2n doubles,
 * V: 8n doubles. */
int npme_gpu_calcv_complex(npme_handle *h, double *V, size_t n,
                           const double *charge, const double *coord);

/* CalcV on device buffers already resident in HBM, enqueued on `stream`
 * (a cudaStream_t; NULL is the default stream, as in CUDA).  Charge and V
 * layouts as above.  Returns after enqueueing; the caller synchronises. */
int npme_gpu_calcv_device(npme_handle *h, double *d_V, const double *d_charge,
                          void *stream);

/* Short-range direct sum alone on device buffers: V = sum_{j != i,
 * r_ij <= Rdir} q_j f_SR(r_ij) and its gradient, no self term, V overwritten.
 * Replaces NPME_PotLaplace_SR_DM_DirectSum_V1 / _SR_Original_DirectSum_V1
 * (src/PotentialLaplace.h:33-44), NPME_PotHelmholtz_SR_DM_DirectSum_V1
 * (src/PotentialHelmholtz.cpp:194) and NPME_PotGenFunc_DirectSum_V1
 * (src/PotentialGenFunc.cpp:140) for the set-up geometry.  Layouts and
 * stream semantics as npme_gpu_calcv_device.  Like the reference's cell-pair
 * loops it evaluates every pair once for both points (built-in kernels and
 * real caller kernels; complex caller kernels and FP64 Helmholtz walk each
 * target's sources), adding the source-side sums with atomics, so repeated
 * calls can differ in the last bits (NPME_PAIRS_ONCE=0 at set-up: one-sided,
 * reproducible). */
int npme_gpu_direct_sum_device(npme_handle *h, double *d_V, const double *d_charge,
                               void *stream);

/* The same short-range direct sum for callers that cannot call cudaMalloc
 * when they need it (for example code inside another framework's pre-reserved
 * memory pool, or a latency-critical loop that must not let an allocation
 * synchronise the device).  No counterpart in the reference.  Allocates
 * nothing: its scratch (the charges gathered into the direct-sum order) is a
 * static 8 MiB device array that every GPU loading the library holds until
 * exit, so at most 2,097,152 points (FP32 real), 1,048,576 (FP32 complex,
 * FP64 real) or 524,288 (FP64 complex); larger handles get NPME_EINVAL.
 * npme_gpu_setup loads the array onto its device (while the caller still
 * allows allocation); each call looks its address up without allocating.
 * Calls share the array: calls that overlap on the GPU race.  The source-side sums of the pair-once walk go to a buffer
 * of the handle that npme_gpu_setup allocated.  Output and arguments as
 * npme_gpu_direct_sum_device. */
int npme_gpu_direct_sum_device_noalloc(npme_handle *h, double *d_V,
                                       const double *d_charge, void *stream);

/* Batched CalcV (no counterpart in the reference, which evaluates one system
 * per call): runs CalcV for `count` set-up handles of the same device in one
 * pass, one kernel launch per stage and launch class (same B-spline order,
 * same pair-kernel coefficients), FFTs per system.  Sizes, kernels, orders and
 * FFT boxes may differ between members.  d_V[i] / d_charge[i] are device
 * buffers laid out as for npme_gpu_calcv_device.  Enqueued on `stream`
 * (NULL: the default stream); the direct sums run on the batch's second
 * stream, joined before the interpolation.  A member handle must not be set
 * up again, nor used in another batch, before npme_gpu_batch_sync returns. */
typedef struct npme_batch npme_batch;
int npme_gpu_batch_create(int device, npme_batch **out);
int npme_gpu_calcv_batch(npme_batch *b, npme_handle *const *handles, int count,
                         double *const *d_V, const double *const *d_charge,
                         void *stream);
int npme_gpu_batch_sync(npme_batch *b);
int npme_gpu_batch_last_error(const npme_batch *b, char *buf, size_t len);
int npme_gpu_batch_destroy(npme_batch *b);

/* Serving queue (the submit/poll surface of a serving deployment; no
 * counterpart in the reference, which evaluates one system per call).  A
 * server owns one device; requests are independent systems, each with its
 * own parameters, geometry and charges.  Requests are admitted in arrival
 * order while the estimated device bytes of the requests in flight stay
 * under hbm_budget; set-up threads prepare them, up to setup_batch in one
 * pass of the set-up kernels, on pooled handles (an idle handle whose device
 * buffers fit, given the request's parameters, else a new one); a dispatch
 * thread runs all prepared requests as one batched CalcV
 * (npme_gpu_calcv_batch), writes each result into the caller's V and
 * completes its ticket.  Thread-safe: any thread may submit, poll or wait.
 * coord, charge and V are host buffers laid out as for npme_gpu_calcv_real /
 * _complex; the caller keeps them alive and unchanged until the ticket is
 * done or failed. */
typedef struct npme_server npme_server;
typedef struct {
  int device;
  int setup_threads;   /* host threads issuing requests' set-ups (default 8) */
  int max_batch;       /* systems per batched CalcV (default 64) */
  size_t hbm_budget;   /* device bytes in flight; 0: half the free memory */
  int pool_capacity;   /* idle handles kept for reuse (default 256; their
                          device bytes stay under pool_bytes) */
  int setup_batch;     /* admitted requests one set-up thread prepares in one
                          pass of the set-up kernels (default 4) */
  size_t pool_bytes;   /* device bytes the idle handles may hold; 0: half the
                          free memory at creation.  A handle keeps the largest
                          buffers it has needed, so a pool that serves a
                          stream of mixed sizes holds more than the requests
                          in flight; one kept below that evicts handles that
                          the next requests then create again.  The server
                          reserves this much of the library's device memory
                          pool at creation (best effort) and keeps it until
                          npme_gpu_server_destroy: growing the pool while
                          kernels run stalls every host thread of the
                          process for tenths of a second */
} npme_server_config;
enum {
  NPME_TICKET_QUEUED = 0,  /* waiting for admission */
  NPME_TICKET_SETUP = 1,   /* being set up */
  NPME_TICKET_READY = 2,   /* set up, waiting for the GPU */
  NPME_TICKET_RUNNING = 3, /* in a batch on the GPU */
  NPME_TICKET_DONE = 4,    /* V written */
  NPME_TICKET_FAILED = 5   /* see npme_ticket_info.error */
};
typedef struct {
  int state;            /* NPME_TICKET_* */
  int status;           /* npme_status of a finished request */
  double t_submit, t_admit, t_ready, t_done; /* seconds since server creation */
  int batch_size;       /* requests in the batch that ran it */
  size_t footprint;     /* estimated device bytes while in flight */
  char error[256];
} npme_ticket_info;
typedef struct {
  unsigned long long submitted, completed, failed;
  unsigned long long batches, batched_requests;
  unsigned long long handles_created, handles_retuned;
  int idle_handles;
  size_t in_flight_bytes, hbm_budget;
  double clock_s;       /* seconds since server creation */
  unsigned long long handles_dropped;  /* let go because the pool was full */
  size_t idle_bytes, pool_bytes;       /* device bytes of the idle handles, limit */
} npme_server_stats;
void npme_gpu_server_default_config(npme_server_config *c);
int npme_gpu_server_create(const npme_server_config *c, npme_server **out);
int npme_gpu_submit(npme_server *s, const npme_params *p, size_t n,
                    const double *coord, const double *charge, double *V,
                    unsigned long long *ticket);
/* state <- NPME_TICKET_* of the ticket */
int npme_gpu_poll(npme_server *s, unsigned long long ticket, int *state);
/* Blocks until the ticket is done or failed (timeout_s < 0: no limit);
 * returns the request's status, or NPME_ETIMEOUT. */
int npme_gpu_wait(npme_server *s, unsigned long long ticket, double timeout_s);
int npme_gpu_ticket_info(npme_server *s, unsigned long long ticket,
                         npme_ticket_info *info);
/* Forgets a finished ticket (NPME_ESTATE while it is in flight). */
int npme_gpu_release_ticket(npme_server *s, unsigned long long ticket);
int npme_gpu_server_stats(npme_server *s, npme_server_stats *st);
/* Completes every submitted request, then frees the server and its handles. */
int npme_gpu_server_destroy(npme_server *s);

/* CalcV_exact: O(N^2) sum with the full kernel (FP64), host buffers. */
int npme_gpu_calcv_exact_real(npme_handle *h, double *V, size_t n,
                              const double *charge, const double *coord);
int npme_gpu_calcv_exact_complex(npme_handle *h, double *V, size_t n,
                                 const double *charge, const double *coord);

/* CalcV_exact (FP64, full kernel, no self term) at m of the set-up points:
 * row t of V (4 doubles, or 4 complex) is the point targets[t], summed over
 * all n charges (charge: n or 2n doubles).  No counterpart in the
 * reference; the grid chooser measures errors with it. */
int npme_gpu_calcv_exact_subset(npme_handle *h, double *V, size_t m,
                                const unsigned int *targets, const double *charge);

/* FFT box for a solve that names none, the job of the reference's
 * NPME_AddMissingKeywords (src/Interface.cpp:256-432), which predicts it
 * with its RSEM error model (src/EstimateParm.cpp).  Here the error is
 * measured instead: starting from a coarse box, the box is refined until the
 * RMS absolute potential error against the exact sum, over up to 4096
 * sampled points, is <= tol (the reference's tol: an absolute RMS error of
 * V), or the FFT arrays would exceed maxFFTmemGB.  p gives every other
 * parameter (its N1..N3 are ignored); on return *out = p with N1..N3 set and
 * *err the measured error.  Uses the GPU (a few solves of the system). */
int npme_gpu_choose_grid(const npme_params *p, size_t n, const double *coord,
                         const double *charge, double tol, double maxFFTmemGB,
                         npme_params *out, double *err);

/* Number of unordered point pairs with 0 < r <= Rdir in the set-up geometry
 * (the work of the direct sum), counted on the device in FP64 over the
 * direct sum's warp groups. */
int npme_gpu_count_pairs(npme_handle *h, unsigned long long *unordered_pairs);

/* Record per-stage CUDA-event timings for subsequent calcv calls (read back
 * with npme_gpu_get_info).  enable = 1: the direct sum stays beside the
 * reciprocal chain on the second stream, so the chain's event pairs include
 * waiting for SMs the direct sum holds; enable = 2: the direct sum starts
 * after the reciprocal chain, so that every stage's event pair times that
 * stage alone (the call takes ~1 % longer); 0: off. */
int npme_gpu_set_timing(npme_handle *h, int enable);

/* CalcV as a CUDA graph (enable = 1, the default): a handle's CalcV launches
 * depend only on its set-up and on the device buffers of the call, so the
 * second npme_gpu_calcv_device (or host-buffer CalcV) with the same buffers
 * after a set-up is captured, and later calls with those buffers launch the
 * captured graph on the caller's stream: one launch instead of ~20 kernel
 * launches and cuFFT calls, which is what bounds CalcV of small systems.  A
 * set-up, npme_gpu_set_params or npme_gpu_set_user_kernel discards the
 * graph; the timing mode and caller-defined kernels always launch plainly.
 * enable = 0: every call enqueues its launches.  No counterpart in the
 * reference (a CPU library). */
int npme_gpu_set_graph(npme_handle *h, int enable);

int npme_gpu_get_info(const npme_handle *h, npme_info *info);

/* Copies the last error message of h (or of the library when h is NULL). */
int npme_gpu_last_error(const npme_handle *h, char *buf, size_t len);

int npme_gpu_destroy(npme_handle *h);

#ifdef __cplusplus
}
#endif

#endif /* NPME_GPU_H */
