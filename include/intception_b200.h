/*
 * intception_b200.h -- C ABI of the B200 (sm_100a) ERI backend.
 *
 * Two groups of entry points:
 *
 * 1. Drop-ins with the exact prototypes the reference generator emits for the
 *    ERI input script (the class "eri" with indices a,b,c,d and auxiliary m).
 *    A host program linked against the generated C99 links against this
 *    library instead; pointers are HOST pointers and the call is synchronous.
 *    The device work runs on the library's own stream on the current device.
 *
 * 2. Batched device entry points (device pointers, a caller stream, status
 *    return) for millions of quartets: class sort, persistent per-class
 *    kernels, optional mixed precision.
 *
 * The drop-ins return void like the reference; intception_b200_last_status()
 * reports the outcome of the last call on the calling thread.
 */
#ifndef INTCEPTION_B200_H
#define INTCEPTION_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------------------------------------------------------
 * 1. Drop-in replacements
 * ------------------------------------------------------------------------- */

/* Replaces intception_integral_eri_abcd_m_cont_cart_main, emitted by the
 * reference into intception_integral_eri_abcd_m_cont_cart.h
 * (argument list: generator/callables/main_source_algorithms/contracted_general.py:42-68;
 * per-index names: generator/wrappers.py:41-143).  Contracted Cartesian
 * (ab|cd) block into output_array with the caller's strides; work_array is
 * accepted for compatibility and not touched. */
void intception_integral_eri_abcd_m_cont_cart_main(
    const double *xa, const double cA[3], const int la, const int na, const int iskipa, const int na_prim,
    const int na_cont, const int iskipa_cont, const double *contract_array_a,
    const double *xb, const double cB[3], const int lb, const int nb, const int iskipb, const int nb_prim,
    const int nb_cont, const int iskipb_cont, const double *contract_array_b,
    const double *xc, const double cC[3], const int lc, const int nc, const int iskipc, const int nc_prim,
    const int nc_cont, const int iskipc_cont, const double *contract_array_c,
    const double *xd, const double cD[3], const int ld, const int nd, const int iskipd, const int nd_prim,
    const int nd_cont, const int iskipd_cont, const double *contract_array_d,
    double *work_array, double *output_array);

/* Replaces intception_integral_eri_abcd_m_cont_cart_work_array_size
 * (contracted_general.py:240-502): same integer result, so callers that size
 * their work arrays with it keep working. */
int intception_integral_eri_abcd_m_cont_cart_work_array_size(
    const int la, const int lb, const int lc, const int ld, const int na_prim, const int nb_prim,
    const int nc_prim, const int nd_prim, const int na_cont, const int nb_cont, const int nc_cont,
    const int nd_cont);

/* Replaces intception_integral_eri_abcd_m_cont_sph_main (spherical variant:
 * generator_options(spherical_transformed=True), generator.py:102-268).  The
 * caller's matrices sph_trans_array_?[icart + isph*ncart] are applied
 * (generator_sph_trans_function.py:69-125). */
void intception_integral_eri_abcd_m_cont_sph_main(
    const double *xa, const double cA[3], const int la, const int na, const int iskipa, const int na_prim,
    const int na_cont, const int iskipa_cont, const double *contract_array_a, const double *sph_trans_array_a,
    const double *xb, const double cB[3], const int lb, const int nb, const int iskipb, const int nb_prim,
    const int nb_cont, const int iskipb_cont, const double *contract_array_b, const double *sph_trans_array_b,
    const double *xc, const double cC[3], const int lc, const int nc, const int iskipc, const int nc_prim,
    const int nc_cont, const int iskipc_cont, const double *contract_array_c, const double *sph_trans_array_c,
    const double *xd, const double cD[3], const int ld, const int nd, const int iskipd, const int nd_prim,
    const int nd_cont, const int iskipd_cont, const double *contract_array_d, const double *sph_trans_array_d,
    double *work_array, double *output_array);

/* Replaces intception_integral_eri_abcd_m_cont_sph_work_array_size. */
int intception_integral_eri_abcd_m_cont_sph_work_array_size(
    const int la, const int lb, const int lc, const int ld, const int na_prim, const int nb_prim,
    const int nc_prim, const int nd_prim, const int na_cont, const int nb_cont, const int nc_cont,
    const int nd_cont);

/* Replaces intception_boys from the emitted boys_function.h
 * (generator_boys_function.py:98-205): f[m*ifskip] = F_m(x), m = nmin..nmax,
 * evaluated by the device Boys module.  For many arguments use
 * intception_b200_boys_batch. */
void intception_boys(double *f, const int ifskip, const int nmin, const int nmax, const double x);

/* Two-index primitive Cartesian classes of the reference's example input
 * script (examples/example_input.py:83-107, generated with contracted=False;
 * argument list: generator/callables/main_source_algorithms/primitive_general.py:31-97,
 * output copy: primitive_general.py:929).  Host pointers, synchronous.
 * output_array[ia*iskipa + ib*iskipb] for the na = (la+1)(la+2)/2 and
 * nb = (lb+1)(lb+2)/2 components (na, nb must equal those counts;
 * intception_b200_last_status() reports IB_ERR_ARG otherwise); 0 <= l <= 6;
 * exponents > 0; work_array is accepted and not touched. */

/* Replaces intception_integral_overlap_2idx_ab_prim_cart_main: (a|b) overlap. */
void intception_integral_overlap_2idx_ab_prim_cart_main(
    const double xa, const double cA[3], const int la, const int na, const int iskipa,
    const double xb, const double cB[3], const int lb, const int nb, const int iskipb,
    double *work_array, double *output_array);

/* Replaces intception_integral_overlap_2idx_ab_prim_cart_work_array_size
 * (primitive_vrr_only_no_auxiliary.py:126-165): ncum(la) * ncum(lb),
 * ncum(l) = (l+1)(l+2)(l+3)/6. */
int intception_integral_overlap_2idx_ab_prim_cart_work_array_size(const int la, const int lb);

/* Replaces intception_integral_nuclear_2idx_ab_m_cC_prim_cart_main: attraction
 * (a| 1/|r-C| |b) to the unit point charge at cC. */
void intception_integral_nuclear_2idx_ab_m_cC_prim_cart_main(
    const double xa, const double cA[3], const int la, const int na, const int iskipa,
    const double xb, const double cB[3], const int lb, const int nb, const int iskipb,
    const double cC[3], double *work_array, double *output_array);

/* Replaces intception_integral_nuclear_2idx_ab_m_cC_prim_cart_work_array_size
 * (primitive_vrr_only_with_auxiliary.py:191-230): 2 (ncum(lb) ncum(la) + la + lb + 1). */
int intception_integral_nuclear_2idx_ab_m_cC_prim_cart_work_array_size(const int la, const int lb);

/* ----------------------------------------------------------------------------
 * Status
 * ------------------------------------------------------------------------- */
#define IB_OK 0
#define IB_ERR_ARG 1       /* invalid argument (l out of range, n mismatch, null pointer) */
#define IB_ERR_CUDA 2      /* CUDA runtime error */
#define IB_ERR_SCRATCH 3   /* a class needed more scratch than reserved */
#define IB_ERR_NODEVICE 4  /* no CUDA device */
#define IB_ERR_TIMEOUT 5   /* a kernel's bounded wait for its own data copies gave up */

/* Status of the last call made on this thread (drop-ins included). */
int intception_b200_last_status(void);
/* Human-readable message for the last failing call on this thread. */
const char *intception_b200_last_error(void);
/* Highest angular momentum per shell the library accepts (6, the reference's global_user_lmax default). */
int intception_b200_lmax(void);

/* ----------------------------------------------------------------------------
 * 2. Batched device API
 * ------------------------------------------------------------------------- */

/* Shell table in device memory (structure of arrays, segmented contraction).
 * prim_coef holds normalised contraction coefficients, as contract_array_?. */
typedef struct {
  const int *shell_l;      /* [nshell] */
  const int *shell_k;      /* [nshell] primitives per shell, 1..64 */
  const int *shell_ptr;    /* [nshell] offset of the first primitive */
  const double *shell_xyz; /* [3*nshell] centres */
  const double *prim_exp;  /* [nprim] */
  const double *prim_coef; /* [nprim] */
  int nshell;
  int nprim;
  int lmax;                /* max shell_l (<= intception_b200_lmax()) */
} intception_b200_basis;

#define IB_PREC_FP64 0  /* every evaluated quartet in FP64 */
#define IB_PREC_MIXED 1 /* FP32 VRR for quartets whose bound < fp32_below, FP64 otherwise */

/* Contracted ERIs for nq quartets.  quartets[4*q+0..3] are shell indices
 * (a,b,c,d); quartet q writes its block at out + out_off[q] with a fastest,
 * index = ia + na*(ib + nb*(ic + nc*id)), na = 2l+1 (spherical, library
 * matrices, m = -l..l) or (l+1)(l+2)/2 (Cartesian).
 * bounds (device, [nq]) is a per-quartet upper bound of |(ab|cd)|, e.g. the
 * Schwarz product of intception_b200_schwarz values; it may be NULL when
 * precision is IB_PREC_FP64 and skip_below is 0.  Quartets with
 * bound < skip_below are screened: their block is written as zeros (error <=
 * bound).  With IB_PREC_MIXED, quartets with bound < fp32_below (and at least
 * skip_below) run the VRR in FP32 (Boys, pair setup, contraction sums, HRR and
 * spherical transforms stay FP64) while accumulating a first-order bound on
 * the FP32 rounding error of the finished block; a quartet whose bound exceeds
 * mixed_tol is recomputed in FP64.  Asynchronous on stream (a cudaStream_t;
 * NULL = the legacy default stream).  Work buffers are reused between calls:
 * calls on different streams must be ordered by the caller. */
int intception_b200_eri_batch(const intception_b200_basis *basis, const int *quartets, const long long *out_off,
                              int nq, int spherical, int precision, const double *bounds, double skip_below,
                              double fp32_below, double mixed_tol, double *out, void *stream);

/* CUDA graph of one intception_b200_eri_batch call (same arguments, fixed
 * device pointers and sizes): the class sort, item build and every class kernel
 * with its side-stream fork/join are captured once and replayed with a single
 * launch.  create runs the batch once eagerly (sizing the work buffers, so the
 * capture allocates nothing) and once under capture; launch replays it on
 * stream; replays read the inputs' current contents.  The graph uses the
 * library's shared work buffers: do not run it concurrently with other batches. */
int intception_b200_eri_graph_create(const intception_b200_basis *basis, const int *quartets,
                                     const long long *out_off, int nq, int spherical, int precision,
                                     const double *bounds, double skip_below, double fp32_below, double mixed_tol,
                                     double *out, void **handle);
int intception_b200_eri_graph_launch(void *handle, void *stream);
int intception_b200_eri_graph_destroy(void *handle);

/* Schwarz factors q[p] = sqrt(max_ij |(ij|ij)|) of the shell pairs
 * pairs[2p], pairs[2p+1] (device pointers), so that |(ab|cd)| <= q_ab q_cd for
 * every function of the quartet; spherical selects the function set the
 * integrals are requested in.  Evaluated with the FP64 batch path on the
 * diagonal quartets, in chunks; returns when q is complete on stream. */
int intception_b200_schwarz(const intception_b200_basis *basis, const int *pairs, int npairs, int spherical,
                            double *q, void *stream);

/* Analytic screening bounds: bounds[q] >= |(ab|cd)| for every element of
 * quartet q (device pointers, asynchronous on stream).  Q_ab sums, over the
 * pair's primitive pairs, a bound on the Coulomb norm of the primitive
 * product (|c_a c_b| exp(-x_a x_b |AB|^2 / zeta) times the norms of
 * (rho + |PA|)^la (rho + |PB|)^lb exp(-zeta rho^2), and for spherical output the
 * transformation's largest coefficient sum; each term in float, widened by
 * 1.001); bounds[q] = Q_ab Q_cd by Cauchy-Schwarz in the Coulomb metric.  No ERI is evaluated: one pass over
 * the primitive pairs, cheap enough to run with every batch (on a random l <= 2
 * batch it keeps 1.3x the quartets Schwarz factors keep at 1e-12).  A value
 * whose true bound is below about 1e-300 may read 0.  A pair with an l above
 * basis->lmax (or outside [0, 6]) gives +inf.  New: the reference has no screening. */
int intception_b200_quartet_bounds(const intception_b200_basis *basis, const int *quartets, int nq, int spherical,
                                   double *bounds, void *stream);

/* Number of library kernels the last intception_b200_eri_batch launched. */
int intception_b200_last_launch_count(void);

/* Waits for the device and returns how many quartets of the last batch had
 * their FP32 result rejected by the error bound and recomputed in FP64 (0
 * unless that batch was IB_PREC_MIXED). */
int intception_b200_last_fp32_rejections(void);

/* Waits for the device and returns how many quartets of the last batch (or
 * drop-in call) the unrolled class kernels handed to the generic kernel
 * because their HRR rounding-error estimate exceeded the tolerance
 * (intception_b200_set_hrr_tol).  New: the reference has no counterpart. */
int intception_b200_last_hrr_redo(void);

/* Blocks of the generic kernel's launch on the current device when heavy
 * quartets are split over thread-block clusters of cluster_size blocks (2 or
 * 4): whole clusters that fit the GPU at once, at most the launch's grid of
 * resident blocks per SM x SMs; cluster_size 1 gives that grid (no clusters).
 * Any other size, or no CUDA device, returns -1.  New: the reference has no
 * counterpart. */
int intception_b200_generic_grid(int cluster_size);

/* Tuning: at most cap lane groups (a power of two; 0 = no cap) share one
 * contracted quartet in the kernel of canonical class cid (cid < 0: every
 * class).  The kernels spread a quartet's primitive quartets over more groups
 * when a class has fewer quartets than the grid has groups; results agree to
 * rounding for every cap.  New: the reference's functions have no such knob. */
int intception_b200_set_slice_cap(int cid, int cap);

/* Primitive screening for the batch entries (intception_b200_eri_batch and its
 * graph form): a primitive quartet whose bound Q_ab Q_cd is below tol is not
 * evaluated.  Q is a Schwarz-type bound on the Coulomb norm of a primitive
 * pair's charge distributions (times the spherical transform's largest
 * coefficient sum), so each skipped primitive quartet moves an element of its
 * block by at most tol; a block moves by at most Ka Kb Kc Kd x tol.  0 (the
 * default) skips only primitive quartets whose prefactor is exactly zero.
 * tol outside [0, 1e-6] returns IB_ERR_ARG.  The drop-in functions never
 * screen.  New: the reference evaluates every primitive quartet. */
int intception_b200_set_prim_tol(double tol);

/* HRR conditioning check of the unrolled class kernels (batch entries and
 * drop-ins).  A pair whose contraction mixes tight and diffuse exponents on
 * both shells has no orientation in which all its primitive pairs keep the
 * horizontal recurrence well conditioned; after contraction each class kernel
 * estimates its HRR rounding error as 32 x 2^-53 x the largest contracted
 * [e0|f0] element times its HRR coefficient bound C(lb,k) |AB|^(lb-k)
 * C(ld,j) |CD|^(ld-j) (k, j its levels above la, lc) and, when that exceeds
 * tol, the quartet is recomputed by the generic kernel, which builds every
 * primitive pair on the shell that conditions its HRR.  Default 1e-13
 * (outputs then agree with an exact evaluation to about 1e-13 on such
 * quartets); 0 switches the check off, and quartets with a pair whose HRR
 * growth bound is large in the class kernels' shell order then go to the
 * generic kernel a priori; tol outside [0, 1e-6] returns IB_ERR_ARG.  New:
 * the reference builds the ket by vertical recurrences on both shells and has
 * no such check. */
int intception_b200_set_hrr_tol(double tol);

/* Tuning: register budget of the kernel of canonical class cid for variant v4
 * (0 FP64 Cartesian, 1 FP64 spherical, 2 FP32 Cartesian, 3 FP32 spherical):
 * the kernel compiled for minb (1, 3, 4 or 5) resident blocks per SM; 0
 * restores the default, the autotuner's table built into the library.  New: the
 * reference has no counterpart. */
int intception_b200_set_class_minb(int cid, int v4, int minb);

/* Tuning: whether the FP32 tier (IB_PREC_MIXED) runs the FP32-VRR kernel of
 * canonical class cid (cid < 0: every class): 1 where the class has one, 0
 * never (that class's FP32-tier quartets are evaluated in FP64), -1 the
 * default built into the library (the classes whose FP32 kernel the autotuner
 * measured faster).  Waits for the device.  New: no reference counterpart. */
int intception_b200_set_class_fp32(int cid, int on);

/* Waits for the device and returns the device status word of the last batch
 * (IB_OK, IB_ERR_ARG for an out-of-range l, IB_ERR_SCRATCH). */
int intception_b200_batch_status(void);

/* Allocation-free variant of intception_b200_eri_batch, for callers that
 * cannot call cudaMalloc (a host framework whose pool allocator owns the device
 * memory, or code that must not trigger the device synchronisation of
 * cudaMalloc/cudaFree).  It has no counterpart in the reference.  Same
 * arguments and output layout as intception_b200_eri_batch with precision
 * IB_PREC_FP64; all quartets go through the block-per-quartet kernel, using
 * file-scope device arrays of fixed size that every GPU loading the library
 * holds until exit: 32 MiB of scratch and descriptors for at most 65536
 * quartets per call (larger nq returns IB_ERR_ARG; IB_ERR_SCRATCH if one
 * quartet of basis->lmax needs more scratch than that).  The first call on a
 * device looks up those arrays and copies the Boys and spherical tables into
 * them (a synchronous copy): make that first call before any stream capture.
 * Calls share the arrays, so calls whose work overlaps on the GPU (unordered
 * streams) race; order them.  Asynchronous on stream (NULL = legacy default).
 * The return value covers the host-side checks and the launches; errors found
 * on the device go to a status word of its own, read with
 * intception_b200_noalloc_status.  A quartet with an l outside
 * [0, basis->lmax] sets IB_ERR_ARG there and, as in intception_b200_eri_batch,
 * is evaluated as (ss|ss) of its shells: the first element of its block is
 * written, nothing else. */
int intception_b200_eri_batch_noalloc(const intception_b200_basis *basis, const int *quartets,
                                      const long long *out_off, int nq, int spherical, double *out, void *stream);

/* Device status word of intception_b200_eri_batch_noalloc on the current
 * device (IB_OK, IB_ERR_ARG for an l out of range, IB_ERR_SCRATCH): waits for
 * stream, then reads the word of the last call.  Allocates nothing; IB_OK
 * before the first call.  No counterpart in the reference. */
int intception_b200_noalloc_status(void *stream);

/* Density digestion (device pointers, asynchronous on stream).  quartets are
 * unique shell quartets (a>=b, c>=d, each pair-pair once), standing for their
 * 8-fold permutation families; blocks/out_off are their Cartesian ERI blocks
 * (a fastest); fofs[s] is the first Cartesian function of shell s; P the
 * symmetric nbf x nbf Cartesian density.  Adds E_J = 1/2 sum P_ij P_kl (ij|kl)
 * to e_out[0] and E_K = -1/4 sum P_ik P_jl (ij|kl) to e_out[1], summed in
 * double-double in a fixed order (the same bits on every run).  Its block
 * partials live in a file-scope device array: calls on one device must be
 * ordered (one stream, or events between streams). */
int intception_b200_jk_energy(const int *quartets, const long long *out_off, int nq, const int *shell_l,
                              const int *fofs, const double *P, int nbf, const double *blocks, double *e_out,
                              void *stream);

/* Nuclear-gradient digestion of one auxiliary batch: for the quartets
 * quartets[qidx[k]], centre pos (0..2) raised (sign +1: shell of l+1 with
 * coefficients 2 alpha c) or lowered (sign -1: l-1), Cartesian blocks at
 * blocks + aux_off[k].  Adds d(E_J + E_K)/dR of centre pos to its atom and the
 * opposite to the atom of centre 3 (translational invariance) in
 * force[3*atom + xyz]; natom <= 4096.  The shell arrays are indexed with the
 * original shell numbers of quartets. */
int intception_b200_jk_force(const int *quartets, const int *qidx, const long long *aux_off, int naux, int pos,
                             int sign, const int *shell_l, const int *fofs, const int *shell_atom, const double *P,
                             int nbf, int natom, const double *blocks, double *force, void *stream);

/* The same gradient from all six auxiliary batches of nq quartets in one pass:
 * batch b = 2 pos + (sign < 0) has its blocks at aux_blocks[b] +
 * aux_off[b][q] for quartet q (aux_off[b][q] = -1: no block, an l = 0 shell
 * at pos for sign -1).  The host arrays aux_off[6] and aux_blocks[6] hold
 * device pointers.  Each original element's density weight is formed once
 * and applied to its raised and lowered partners of every centre and
 * direction; the result equals the six intception_b200_jk_force calls. */
int intception_b200_jk_force_all(const int *quartets, int nq, const long long *const *aux_off,
                                 const double *const *aux_blocks, const int *shell_l, const int *fofs,
                                 const int *shell_atom, const double *P, int nbf, int natom, double *force,
                                 void *stream);

/* Batched two-index primitive integrals (no counterpart in the reference,
 * which emits one call per pair): pair i of n has exponents xa[i], xb[i],
 * centres ca[3i..], cb[3i..], angular momenta la[i], lb[i] <= lmax <= 6 and,
 * for IB_TWOIDX_NUCLEAR, the charge position cc[3i..] (cc may be NULL for
 * overlap).  Its block goes to out + off[i], a fastest
 * (out[off[i] + ia + na*ib]).  Device pointers; asynchronous on stream (NULL =
 * legacy default).  A pair with l outside [0, lmax] or an exponent <= 0 is
 * skipped and IB_ERR_ARG is stored in *status (a device int, may be NULL). */
#define IB_TWOIDX_OVERLAP 0
#define IB_TWOIDX_NUCLEAR 1
int intception_b200_twoidx_batch(int kind, int n, int lmax, const double *xa, const double *ca, const int *la,
                                 const double *xb, const double *cb, const int *lb, const double *cc,
                                 const long long *off, double *out, int *status, void *stream);

/* Testing the two-index kernel's bounded waits (no counterpart in the
 * reference): the next intception_b200_twoidx_batch call announces chunk
 * `chunk`'s bytes (IB2 chunks of 512 pairs, fetched by bulk copies when every
 * input array is 16-byte aligned) on its barrier but issues no copy for it,
 * and polls wait_iters times (1 .. 1 << 22) before it gives up.  The block
 * owning that chunk then stores IB_ERR_TIMEOUT in *status, waits for its other
 * copies in flight and returns without writing its pairs.  One-shot. */
int intception_b200_twoidx_test_stall(long long chunk, int wait_iters);

/* The library's Cartesian->spherical matrix for l (host memory,
 * T[icart + isph*ncart], ncart x (2l+1)). */
int intception_b200_sph_matrix(int l, double *T);

/* F_m(x[i]) for m = 0..nmax into f[i*(nmax+1) + m]; device pointers; NULL
 * stream = the legacy default stream. */
int intception_b200_boys_batch(const double *x, int n, int nmax, double *f, void *stream);

/* Block until the library stream is idle. */
int intception_b200_synchronize(void);

/* Diagnostics: FP64 (fp64 != 0) or FP32 FMA throughput of the current device
 * in FLOP/s, from a kernel of independent FMA chains (iters x 128 FMAs per
 * thread); the roofline denominator of the ERI kernels. */
int intception_b200_fma_peak(int fp64, int iters, double *flops_per_second);

#ifdef __cplusplus
}
#endif
#endif /* INTCEPTION_B200_H */
