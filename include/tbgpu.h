/*
 * tbgpu.h -- C ABI of the B200 tight-binding eigensolver (libtbgpu.so).
 *
 * The three seams of NEMO-3D's electronic-structure hot path are replaced:
 *
 *   Hamiltonian build   setup_hamiltonian + first Hmult_spds_complete
 *                       (nemo3d/src/base/ham3d_final.c:731,
 *                        nemo3d/src/base/h_cvectr_mult.c:1194-1196)
 *                       -> tbgpu_ctx_create + tbgpu_build_hamiltonian
 *   H*x                 matvect_mult, the "matmul" function pointer
 *                       (nemo3d/src/base/h_cvectr_mult.c:205-258,
 *                        eigen/include/lanczos.h:287,336,389)
 *                       -> tbgpu_matvect_mult (same signature)
 *   Lanczos driver      eigensolve_lanczos (eigen/src/lanczos.c:1823-2089,
 *                        eigen/include/lanczos.h:365-391)
 *                       -> tbgpu_eigensolve_lanczos
 *
 * All pointers are plain host pointers unless the name ends in _dev (device
 * pointers on the context's CUDA device; device vectors must start on a
 * 16-byte boundary, as cudaMalloc's do, else TBGPU_E_ARG).  Complex vectors are interleaved
 * (re, im) doubles, layout-compatible with nml_dcscalar {double r, i}, in the
 * reference's order: index = atom * NBasisStates + orbital, spin-up orbitals
 * first (nemo3d/src/base/ham3d_final.c:547-620).
 *
 * Error convention: functions return TBGPU_OK (0) or a negative TBGPU_E_*
 * code; a positive return of tbgpu_eigensolve_lanczos is the number of
 * eigenvalues found.  tbgpu_last_error() repeats the last failure code of the
 * calling thread and tbgpu_error_string() describes it.  The reference aborts
 * via die()/error() instead (eigen/src/lanczos.c:270-296); nothing here exits
 * the process.  A context is not re-entrant; distinct contexts are
 * independent.  Every call runs on the context's CUDA stream.
 */
#ifndef TBGPU_H
#define TBGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TBGPU_OK 0
#define TBGPU_E_ARG (-1)          /* invalid argument or size                */
#define TBGPU_E_CUDA (-2)         /* a CUDA call failed                       */
#define TBGPU_E_NOMEM (-3)        /* device allocation failed                 */
#define TBGPU_E_MATERIAL (-4)     /* a bond has no material parameter set     */
#define TBGPU_E_STATE (-5)        /* call out of order (e.g. H not built)     */
#define TBGPU_E_UNSUPPORTED (-6)  /* option not supported by this build       */
#define TBGPU_E_NUMERIC (-7)      /* breakdown (beta = 0, zero pivot, NaN)    */
#define TBGPU_E_TIMEOUT (-8)      /* a bounded device-side wait ran out       */

/* band models: orbitals per spin x spins (mb_ham_spds_micro2.h:43-48) */
#define TBGPU_SP3S 1          /* 5 x 1: spin-up block of Bands_10_sp3ss_spin   */
#define TBGPU_SP3S_SO 2       /* 5 x 2: Bands_10_sp3ss_spin                    */
#define TBGPU_SP3D5S 3        /* 10 x 1: Bands_10_sp3d5ss_nospin               */
#define TBGPU_SP3D5S_SO 4     /* 10 x 2: Bands_20_sp3d5ss_spin                 */

#define TBGPU_NPAR 68         /* 35 mb_pv + 33 mb_strain after param_init      */

typedef struct {
  double r, i;
} tbgpu_dcomplex; /* layout of nml_dcscalar */

typedef struct tbgpu_ctx tbgpu_ctx;

/* Geometry: a dense grid of zincblende conventional cells, cell (i,j,k)
 * row-major with k fastest (the cell order of geo_struct::FillFirstShape,
 * nemo3d/src/base/ham3d.c:745-900), 8 sites per cell (sites 0..3 cations,
 * 4..7 anions, nemo3d/src/base/Cell.c:185-210).  Replaces geo_struct's
 * AtomType / l_m_2_atomdsp (nemo3d/src/base/geo_struct.c:2109-2131). */
typedef struct {
  int nx, ny, nz;
  int periodic[3];            /* periodic axes (Gamma point only)            */
  double lattice[3];          /* a_x, a_y, a_z of the device (nm)            */
  const unsigned char *type;  /* [nx*ny*nz*8] species id, 0 = no atom        */
  const double *dsp;          /* [nx*ny*nz*8*3] displacement (nm) or NULL    */
} tbgpu_geom;

/* Physics options and parameters (ExecParam.Phys / ElCalc of the XML deck). */
typedef struct {
  int band_model;             /* TBGPU_SP3S ... TBGPU_SP3D5S_SO              */
  int include_strain;         /* include_strain_in_Hamiltonian               */
  int passivate;              /* SurfacePassivation == PassivateDanglingBond */
  double dangling_shift;      /* DanglingBondEnergyShift (eV)                */
  int nspecies;               /* species ids 0..nspecies-1                   */
  const double *par;          /* [nspecies][nspecies][TBGPU_NPAR], (c, a)    */
  const unsigned char *par_ok;/* [nspecies][nspecies]                        */
} tbgpu_model;

/* param_init for one material set (nemo3d/src/base/mat3d.c:133-307 with
 * param_sp3s_2_sp3d5s, nemo3d/src/ham/mb_ham_spds_micro.c:2984-3026):
 * sp3s_family = 1 for a 15-entry sp3s* mb_pv.  out[TBGPU_NPAR]. */
int tbgpu_prepare_params(int sp3s_family, int include_strain,
                         const double *mb_pv, const double *mb_strain,
                         double ev_offset, double a0, double *out);

/* Create a context on the current CUDA device; geometry and tables are copied
 * (host pointers).  tbgpu_ctx_create_dev takes device pointers for type/dsp. */
int tbgpu_ctx_create(const tbgpu_geom *geom, const tbgpu_model *model,
                     tbgpu_ctx **out);
int tbgpu_ctx_create_dev(const tbgpu_geom *geom_dev, const tbgpu_model *model,
                         tbgpu_ctx **out);
int tbgpu_ctx_destroy(tbgpu_ctx *ctx);

/* Use a caller-owned CUDA stream (cudaStream_t passed as void*). */
int tbgpu_set_stream(tbgpu_ctx *ctx, void *stream);

/* Topology + Slater-Koster assembly on the GPU (replaces Hmult_spds_col's
 * store pass, nemo3d/src/base/h_cvectr_mult.c:1134-1886). */
int tbgpu_build_hamiltonian(tbgpu_ctx *ctx);

long tbgpu_num_atoms(const tbgpu_ctx *ctx);
long tbgpu_dimension(const tbgpu_ctx *ctx); /* complex length n_atoms * nb */

/* Drop-in for the reference's matmul pointer (h_cvectr_mult.c:205):
 * argList[0] = (int*)ctx, argList[1] = (int*)&shift (double), y = (H-shift)x
 * over host vectors of length tbgpu_dimension(ctx).  On failure y is left
 * unspecified and tbgpu_last_error() is set. */
void tbgpu_matvect_mult(const int **argList, tbgpu_dcomplex *y,
                        const tbgpu_dcomplex *x);
/* The same with device vectors (complex, interleaved doubles, 16-byte
 * aligned): argList as above; asynchronous on the context stream; failures
 * through tbgpu_last_error(). */
void tbgpu_matvect_mult_dev(const int **argList, double *y_dev, const double *x_dev);

/* Precision of the stored Hamiltonian: 64 (default) or 32 bits, set before
 * tbgpu_build_hamiltonian.  32 is the reference's HamMemorySave build
 * (nemo3d/src/base/HamZincBlende.h:51-66, Hmult_stored.c:629, 910): the
 * bond blocks and on-site records are rounded to float after assembly and
 * widened again inside H*x, whose arithmetic and vectors stay double.  Half
 * the Hamiltonian's bytes; entries carry float rounding (~6e-8 relative). */
int tbgpu_set_ham_precision(tbgpu_ctx *ctx, int bits);

/* Storage of the bond blocks, set before tbgpu_build_hamiltonian: 0 (default)
 * assembles and stores them once (the reference's HamCompute=SparseStore,
 * XMLtoC/apps/ioNemo3D/src/ElAlg_struct.H:25);
 * 1 recomputes each block inside every H*x from the geometry and the
 * parameters (HamCompute=Recompute, Hmult_spds_col multiplying on the fly,
 * nemo3d/src/base/h_cvectr_mult.c:1134-1886): only the on-site records are
 * stored, for structures whose blocks would not fit in device memory, at the
 * price of the Slater-Koster arithmetic in every product.  Not combined with
 * the 32-bit store (TBGPU_E_UNSUPPORTED at build); tbgpu_hx_dot_noalloc
 * refuses recompute contexts with TBGPU_E_UNSUPPORTED. */
int tbgpu_set_ham_storage(tbgpu_ctx *ctx, int recompute);

/* Precision of the Lanczos vectors, set before tbgpu_build_hamiltonian: 64
 * (default) or 32.  32 is the mixed-precision solve (no counterpart in the
 * reference): it runs on the 32-bit store, tbgpu_set_ham_precision(ctx, 32),
 * or on the recompute storage, tbgpu_set_ham_storage(ctx, 1) (float
 * Slater-Koster elements from double geometry), with any model; else
 * TBGPU_E_UNSUPPORTED at build.  The
 * recurrence vectors are complex float and H*x accumulates in float, while
 * alpha, beta, their reductions, the tridiagonal eigenvalues, the
 * convergence test and the eigenvector accumulation stay double.  The
 * eigenvectors a solve returns are then refined in double: H*v with the
 * double-precision recompute product (bit-identical blocks to the stored
 * assembly), a Rayleigh-Ritz step over groups of up to 8 vectors, and the
 * refined eigenvalues replace the Lanczos ones; the residual
 * ||H v - lambda v|| and the change of each eigenvalue are returned by
 * tbgpu_get_state_errors.  Eigenvalues without a requested vector keep the
 * float recurrence's accuracy.  Not with Bloch phases (TBGPU_E_UNSUPPORTED
 * at solve). */
int tbgpu_set_lanczos_precision(tbgpu_ctx *ctx, int bits);

/* Per state of the last solve of a mixed-precision context, for the n
 * states that had eigenvectors: residual[i] = ||H v_i - lambda_i v_i|| (eV,
 * unit v_i) and delta[i] = lambda_i(refined) - lambda_i(Lanczos).  Either
 * pointer may be NULL.  Returns the number of states written (<= cap). */
int tbgpu_get_state_errors(const tbgpu_ctx *ctx, int cap, double *residual, double *delta);

/* Bloch vector for periodic structures (geo_struct::phasePeriodic,
 * nemo3d/src/base/geo_struct.h:811-826, used by Hmult_stored.c:386-437): a
 * bond that crosses the periodic boundary by images w (-1/0/+1 per axis)
 * carries exp(i*ph), ph = -pi*(w.k - 2*int(0.5*w.k)), k in the reference's
 * units.  k = NULL or (0,0,0) is the Gamma point.  Call after
 * tbgpu_build_hamiltonian; applies to every later H*x and solve.  Away from
 * Gamma, H*x runs the lane-gather kernel. */
int tbgpu_set_bloch_k(tbgpu_ctx *ctx, const double *k);

/* Start vector for the solves (the reference's lanczos_initialize /
 * initStartVect with ReadFile, nemo3d/src/base/eigsys3d_par.c:113-215,
 * nemo3d/src/io/i_3dout_files.c:2292): a host vector of tbgpu_dimension(ctx)
 * complex entries, copied to the device and used by tbgpu_eigensolve_lanczos
 * and tbgpu_eigensolve_lanczos_dev whenever they are called with a NULL
 * start; NULL clears it.  After the build (TBGPU_E_STATE before). */
int tbgpu_set_start_vector(tbgpu_ctx *ctx, const tbgpu_dcomplex *r_0);

/* y = (H - shift) x on device vectors (asynchronous on the context stream). */
int tbgpu_hx_dev(tbgpu_ctx *ctx, double shift, const double *x_dev,
                 double *y_dev);

/* The mixed-precision product: y = (H - shift) x on complex-float device
 * vectors ({float re, im} per entry), accumulated in float, over the 32-bit
 * store or recomputed in float (recompute storage), any model: the H*x of
 * a tbgpu_set_lanczos_precision(ctx, 32) solve; no counterpart in the
 * reference.  At the Gamma point only; else TBGPU_E_UNSUPPORTED. */
int tbgpu_hx_dev_f32(tbgpu_ctx *ctx, double shift, const float *x_dev, float *y_dev);

/* Y_v = (H - shift) X_v for a block of p <= 8 device vectors stored one
 * after the other ([p][dimension] complex): the block product the block
 * Lanczos driver needs (the reference's matmat_mult,
 * nemo3d/src/base/h_cmat_mult.c:21).  For the 10-orbital models at the Gamma
 * point one launch applies each staged bond block to all p vectors;
 * otherwise it runs p H*x launches.  Asynchronous on the context stream. */
int tbgpu_hx_block_dev(tbgpu_ctx *ctx, int p, double shift, const double *x_dev,
                       double *y_dev);

/* Lanczos eigensolver with the semantics of eigensolve_lanczos
 * (eigen/src/lanczos.c:1823-2089): plain Lanczos, convergence test every
 * ConvCheckSkipRate iterations after ConvCheckStartIter on the last two
 * components of the tridiagonal eigenvector (lanczos.c:764-996), degenerate
 * and ghost values dropped at resolution 100*tolerance, windows
 * (emin1,emax1] and (emin2,emax2].  r_0: host start vector, or NULL for
 * the one set by tbgpu_set_start_vector (normalised here,
 * as lanczos_initialize does, eigsys3d_par.c:113-215).  values[>= imax]
 * receives the eigenvalues ascending; conv_iterations (optional) the
 * iteration at which each converged; *iterations the iteration count.  If
 * vectors != NULL, the eigenvectors of the first max_vectors eigenvalues are
 * rebuilt by a second Lanczos pass (eigenvectorsLanczos, lanczos.c:1364-1689)
 * into vectors[max_vectors][dimension].  Returns the number of eigenvalues
 * found or a negative error code. */
int tbgpu_eigensolve_lanczos(tbgpu_ctx *ctx, int ConvCheckStartIter,
                             int ConvCheckSkipRate, int imax, int requested1,
                             int requested2, double emin1, double emax1,
                             double emin2, double emax2, double tolerance,
                             const tbgpu_dcomplex *r_0, double *values,
                             int *conv_iterations, int *iterations,
                             tbgpu_dcomplex *vectors, int max_vectors);

/* Same with the start vector and the eigenvectors in device memory. */
int tbgpu_eigensolve_lanczos_dev(tbgpu_ctx *ctx, int ConvCheckStartIter,
                                 int ConvCheckSkipRate, int imax,
                                 int requested1, int requested2, double emin1,
                                 double emax1, double emin2, double emax2,
                                 double tolerance, const double *r0_dev,
                                 double *values, int *conv_iterations,
                                 int *iterations, double *vectors_dev,
                                 int max_vectors);

/* Eigenvalues in (vl, vu] of an n x n complex Hermitian band matrix with kd
 * subdiagonals, lower band storage as LAPACK's UPLO='L' (column j holds rows
 * j..j+kd at ab[(j*(kd+1) + i-j)*2 + {0,1}], interleaved complex): the
 * solve the block Lanczos driver uses in place of zhbevx RANGE='V'
 * (eigen/src/lanczos_blk.c:891-991).  Host only.  w receives up to cap
 * values ascending; returns how many lie in the window. */
int tbgpu_band_eigenvalues(int n, int kd, const double *ab, double vl, double vu,
                           double abstol, double *w, int cap);

/* Block Lanczos eigenvalues with the semantics of eigensolve_blk_lanczos
 * (eigen/src/lanczos_blk.c:2145-2540, block_lanczos_blocktridiagonal
 * 1412-1678): block size p (1..8), start block r0[p][dimension] (the
 * reference draws it with rand(); here the caller supplies it), the band
 * matrix solved in (emin1,emax1] and (emin2,emax2] every ConvCheckSkipRate
 * steps after ConvCheckStartIter, convergence by Method 4 (values that
 * repeat between checks to `tolerance`), stop when both windows have their
 * requested counts, after max_no_success fruitless steps (<= 0: no limit)
 * or at imax steps.  values[>= requested1 + requested2] receives the
 * eigenvalues ascending; found_vb / found_cb the counts per window;
 * *iterations the block steps.  Returns the number of eigenvalues or a
 * negative error (TBGPU_E_NUMERIC when a block loses rank: deflation is not
 * supported).  If vectors != NULL the eigenvectors of the first max_vectors
 * eigenvalues (ascending) are rebuilt by a second pass
 * (eigenvectorsBlockLanczos, lanczos_blk.c:1857-2145) from eigenvectors of
 * the band matrix found by inverse iteration, into vectors[k][dimension];
 * vectors of equal eigenvalues are made orthogonal. */
int tbgpu_eigensolve_blk_lanczos(tbgpu_ctx *ctx, int ConvCheckStartIter,
                                 int ConvCheckSkipRate, int imax, int requested1,
                                 int requested2, double emin1, double emax1,
                                 double emin2, double emax2, double tolerance,
                                 int p, int max_no_success,
                                 const tbgpu_dcomplex *r0, double *values,
                                 int *found_vb, int *found_cb, int *iterations,
                                 tbgpu_dcomplex *vectors, int max_vectors);
int tbgpu_eigensolve_blk_lanczos_dev(tbgpu_ctx *ctx, int ConvCheckStartIter,
                                     int ConvCheckSkipRate, int imax,
                                     int requested1, int requested2,
                                     double emin1, double emax1, double emin2,
                                     double emax2, double tolerance, int p,
                                     int max_no_success, const double *r0_dev,
                                     double *values, int *found_vb,
                                     int *found_cb, int *iterations,
                                     double *vectors_dev, int max_vectors);

/* Block dots G = X^H Y of two blocks of p (1..8) complex vectors on the
 * tensor cores, to double precision: the p x p inner products of the block
 * QR and of Q^H W in every block Lanczos step (eigen/src/lanczos_blk.c:
 * 150-219, 273-357).  x_dev, y_dev: p vectors of n2 complex entries back to
 * back (interleaved re, im; 16-byte aligned), device memory.  G (host) gets
 * the row-major p x p complex matrix, G[2(ip+j)] + i G[2(ip+j)+1] = x_i^H y_j.
 * The entries are cut into eight 7-bit integer slices (56 bits) with one
 * exponent per 256 entries and vector part, and multiplied by tcgen05.mma
 * kind::i8 with int32 accumulators; per entry the error is below 2^-50 of
 * max|x| max|y| over its 256-entry chunk (a double dot: 2^-53 of each
 * product, plus the rounding of its sums).  Runs on the
 * context's stream and synchronises it; status word checked (TBGPU_E_TIMEOUT
 * when a tensor-core wait ran out). */
int tbgpu_block_dots_dev(tbgpu_ctx *ctx, int p, const double *x_dev, const double *y_dev,
                         long n2, double *G);

/* Which kernel forms the block dots of tbgpu_eigensolve_blk_lanczos(_dev):
 * 0 (default) the double-precision CUDA-core kernel, 1 the tensor-core kernel
 * of tbgpu_block_dots_dev.  TBGPU_E_ARG for another mode. */
int tbgpu_set_block_dots(tbgpu_ctx *ctx, int mode);

/* Mixed-precision Lanczos (tbgpu_set_lanczos_precision(32)): floor of the
 * bound on the last two components of a tridiagonal eigenvector below which
 * the convergence test accepts its Ritz value (the test of lanczos.c's
 * eigenvaluesLanczos uses the solve's tolerance; the complex-float
 * recurrence cannot drive those components below its rounding level, so
 * with a tolerance under that level it accepts values late or not at all).
 * The accepted values are refined in double precision (Rayleigh-Ritz over
 * the double product) and tbgpu_get_state_errors reports their residuals.
 * floor < 1; 0 (default) keeps the tolerance; a negative floor sets it at
 * every check to 2^-24 times the Gershgorin bound of the
 * tridiagonal matrix so far (max_i |alpha_i| + |beta_i| + |beta_i-1|), the
 * rounding level of the complex-float vectors relative to ||H||.  The bound
 * used is max(tolerance, floor).  Double-precision solves ignore it.
 * TBGPU_E_ARG for floor >= 1, NaN or -infinity. */
int tbgpu_set_mixed_acceptance(tbgpu_ctx *ctx, double floor);

/* The Lanczos solves take their per-solve device buffers (the recurrence's
 * vectors, the eigenvector pass's checkpoints and segment rings: tens of GB
 * for a 2M-atom dot) from one memory pool per device that keeps its memory
 * mapped after the solve, so that later solves in the process reuse it
 * instead of mapping and unmapping it again (which took up to seconds of
 * host time per solve).  This returns the memory the pools hold but no
 * solve uses to the device; call it once the solves' streams have
 * finished.  No counterpart in the reference (its buffers come from
 * malloc). */
int tbgpu_release_solver_memory(void);

/* Tridiagonal matrix of the last solve: alpha[n], beta[n] (n <= cap). */
int tbgpu_get_tridiagonal(const tbgpu_ctx *ctx, double *alpha, double *beta,
                          int cap);

/* The saved state of eigensolve_lanczos (eigen/src/lanczos.c:1692-1809):
 * tridiagonal matrix file (int iterations, int processors, double
 * t[2*iterations], t[2i] = alpha_i, t[2i-1] = beta_{i-1}) and eigenvalue file
 * (int n, double value[n]), native endian.  Reading a matrix file keeps
 * iterations - 200 of what is stored, as the reference's
 * restoreTridiagonalMatrix does (lanczos.c:1765), and returns that count
 * (alpha[i], beta[i] for i < min(count, cap); beta couples i and i+1).
 * Reading an eigenvalue file returns n.  Host only; TBGPU_E_ARG when a file
 * cannot be opened or is short. */
int tbgpu_write_tridiagonal_file(const char *path, const double *alpha, const double *beta,
                                 int iterations, int processors);
int tbgpu_read_tridiagonal_file(const char *path, int cap, double *alpha, double *beta,
                                int *processors);
int tbgpu_write_eigenvalue_file(const char *path, const double *values, int n);
int tbgpu_read_eigenvalue_file(const char *path, int cap, double *values);

/* Eigenvectors of nvalues eigenvalues from a given tridiagonal matrix of
 * `iterations` Lanczos steps (alpha[iterations], beta[iterations - 1]) and
 * the start vector r_0 it was built from -- the restoreState path of
 * eigensolve_lanczos (lanczos.c:1912-1955, 2022-2057): no first pass, the
 * recurrence is rerun from r_0 for `iterations` steps and every value's Ritz
 * vector uses the whole matrix.  Values are taken in ascending order;
 * min(nvalues, max_vectors) vectors (host, complex) are written and that
 * count returned. */
int tbgpu_eigenvectors_from_tridiagonal(tbgpu_ctx *ctx, int iterations, const double *alpha,
                                        const double *beta, int nvalues, const double *values,
                                        const tbgpu_dcomplex *r_0, tbgpu_dcomplex *vectors,
                                        int max_vectors);

/* Export for parity tests (tbgpu_export_pattern mirrors the topology of
 * get_total_hamiltonian_dimension_and_offsets / remove_few_bonded_atoms /
 * FindSurfaceAtoms): atom_site[n_atoms] site index of each atom,
 * nbr[n_atoms*4] neighbour atom or -1 in Cell.c nnmap order,
 * surface[n_atoms] 1 for atoms with fewer than four neighbours. */
int tbgpu_export_pattern(const tbgpu_ctx *ctx, int *atom_site, int *nbr,
                         unsigned char *surface);

/* Export the assembled H: onsite[n_atoms][nb][nb] complex (interleaved) and
 * blocks[n_atoms][4][norb][norb] real, nonzero for cation atoms only,
 * blocks[c][a] = <anion orbital a | H | cation orbital c>. */
int tbgpu_export_hamiltonian(const tbgpu_ctx *ctx, double *onsite,
                             double *blocks);

/* y = (H - shift) x and *dot_dev = Re<x, y> on device buffers (x, y of
 * tbgpu_dimension(ctx) complex entries, dot_dev one double), allocating
 * nothing.  No counterpart in the reference: it serves callers that cannot
 * let the library allocate -- device memory handed entirely to their own pool
 * allocator, or iteration loops that cannot take the device-wide
 * synchronisation of cudaMalloc/cudaFree.  The reduction scratch is a fixed
 * array inside the library (2048 block partials + a counter, 16,640 bytes
 * per device, held until exit); launches needing more than 2048 blocks are
 * refused with TBGPU_E_ARG (10-orbital models: never at the Gamma point,
 * above 49,152 atoms with a Bloch vector set; 5-orbital models: above
 * 98,304 atoms).  Every call shares that array: calls that overlap on the GPU
 * race and must be serialised by the caller.  The first call on a device
 * looks up the array's address with that device current; make that first
 * call before any stream capture.  The context's device must be current. */
int tbgpu_hx_dot_noalloc(tbgpu_ctx *ctx, double shift, const double *x_dev,
                         double *y_dev, double *dot_dev);

/* H*x kernel: 0 = default (warp-staged kernel, 14 warps x 1 stage per SM,
 * each cation's block run by one bulk copy (TMA), the other pieces by
 * 16-byte cp.async, for the 10-orbital models; lane-gather kernel
 * otherwise),
 * 1 = lane-gather kernel for every model, 2 = warp-staged kernel with
 * 7 warps x 2 stages, 3 = two-cell unit kernel (bulk copies of each unit's
 * contiguous pieces; 10-orbital models with the 64-bit store at the Gamma
 * point, else as 0), 4 = the default kernel with every piece, the cation
 * block runs included, by 16-byte cp.async, 5 = one lane per (atom, spin)
 * with block rows loaded straight to registers (10-orbital models with a
 * stored Hamiltonian at the Gamma point, else as 0), 6 = the same lane
 * mapping on a pencil-interleaved copy of the Hamiltonian (every quantity
 * stored with the k index of its cell fastest, so a warp's loads are
 * contiguous; the solves keep their Lanczos vectors in that layout, these
 * products permute the caller's vectors around the kernel; Gamma point, not
 * in batched solves, else as 0), 7 = variant 6 with each warp's next bond's
 * block rows double-buffered in shared memory by 16-byte cp.async copies
 * while it computes the current one (32-bit store, spin-orbit models, closed
 * z boundary and nz a multiple of 16; else as 6), 8 and 9 = the
 * lane-gather kernel of variant 1 with 4 and 2 warps per block instead of
 * 8 (the block size sets each block's staging array and so the blocks and
 * warps an SM holds), for every model.  Variants 0, 2, 3 and 4 give the same
 * y bit for bit, and so do 6 and 7, and 1, 8 and 9; 1, 5 and 6 sum in their
 * own orders (equal to rounding).  For 5-orbital models and Bloch phases,
 * 0 to 7 all run the lane-gather kernel with 8 warps per block. */
int tbgpu_set_spmv_variant(tbgpu_ctx *ctx, int variant);

/* Autotuner: times the H*x variants that are distinct kernels for the built
 * context (0 to 6, 8 and 9 for the 10-orbital models with the 64-bit store
 * at the Gamma point; 0, 1, 5, 6, 8, 9 and, where it applies, 7 with the
 * 32-bit store; 0, 8 and 9 for 5-orbital models and Bloch phases; only 0
 * with recompute storage), reps launches each with the fused
 * Lanczos dot after two untimed ones (CUDA events on the context stream;
 * two temporary device vectors), selects the fastest (ties: the lower
 * number) and returns it with its time per launch.  Synchronous. */
int tbgpu_autotune_spmv(tbgpu_ctx *ctx, int reps, int *variant_out, double *ms_out);

/* Lanczos for many independent dots at once (no counterpart in the
 * reference, which solves one structure per run): the context's grid holds
 * ndots dots side by side along x, dot d in the cells i in [dot_cells[d],
 * dot_cells[d+1]) (ndots+1 ascending boundaries), separated by empty cells so
 * that no bond joins two dots (TBGPU_E_ARG otherwise).  Each dot runs the
 * reference's recurrence and convergence test (eigensolve_lanczos) on its own
 * segment of the vectors with its own windows emin1[d]..emax2[d]; all dots
 * iterate together, each iteration one product launch for all dots and
 * segmented reductions, one check interval captured as a CUDA graph.
 * r0_dev: the packed start vector (each dot's segment is normalised on its
 * own).  values: [ndots][values_stride] ascending per dot; found[d],
 * iterations[d] per dot.  vectors_dev ([max_vectors][dimension], or NULL):
 * vector e holds every dot's e-th eigenvector in the dot's segment
 * (max_vectors <= 16).  With tbgpu_set_lanczos_precision(ctx, 32) the dots'
 * eigenpairs are refined in double as in tbgpu_eigensolve_lanczos, state
 * errors [ndots][max_vectors] through tbgpu_get_state_errors.  Returns the
 * total number of values, or a negative error code. */
int tbgpu_eigensolve_lanczos_batched(tbgpu_ctx *ctx, int ndots, const int *dot_cells,
                                     int ConvCheckStartIter, int ConvCheckSkipRate, int imax,
                                     int requested1, int requested2, const double *emin1,
                                     const double *emax1, const double *emin2,
                                     const double *emax2, double tolerance,
                                     const double *r0_dev, double *values, int values_stride,
                                     int *found, int *iterations, double *vectors_dev,
                                     int max_vectors);

/* Result files in the reference's <HDR> format (nemo3d/src/io/fileformat.c:
 * 182-204), readable by its post-processing tools.
 * tbgpu_write_eigenvalues: the nd_Ek file (writeEigenvalues,
 * nemo3d/src/io/i_3dout_files.c:1886-1975): mode 'i' empties the file, 'a'
 * appends n records {kx, ky, kz, E} and rewrites the header's count.
 * tbgpu_write_eigenvector: one nd_evec file (writeEigenvector,
 * i_3dout_files.c:1342-1357) with records {wf.r, wf.i} for every basis state
 * of the context; crystal_structure is the reference's enum (2: zincblende).
 * Host code; TBGPU_OK, or TBGPU_E_ARG for an I/O error or a malformed file. */
int tbgpu_write_eigenvalues(const char *path, char mode, const double *k, int n,
                            const double *E);
int tbgpu_write_eigenvector(const tbgpu_ctx *ctx, const char *path,
                            const tbgpu_dcomplex *wf, int crystal_structure);

/* Keating valence-force-field strain (the reference's min_estrain with
 * StrainModel = VFF_keating: calc_estrain, nemo3d/src/base/strain3d.c:
 * 1361-2080, minimised by macoptII_par, NEMO_3D/eigen/src/macopt_par.c:
 * 121-475).  Both act on a context before tbgpu_build_hamiltonian
 * (TBGPU_E_STATE after it).  vff: [nspecies][nspecies][3] = (a0 nm, alpha,
 * beta) per species pair, symmetric (the reference's amat, alpha, beta); a
 * pair present in the structure with a0 <= 0 is TBGPU_E_MATERIAL.
 * Displacements are per site, [nx*ny*nz*8][3] nm like tbgpu_geom.dsp.
 * tbgpu_vff_energy: the energy at the context's displacements (zero when it
 * has none) and, if grad is not NULL, the reference's gradient dp (the
 * bond-stretching term counted from each bond's atoms for the energy, moving
 * only the vertex atom in the gradient).  tbgpu_vff_relax: macopt from the
 * context's displacements with the reference's boundary conditions bc
 * (0 AllFree, 1 FixOne, 2 FixSurfaceAll, 3 FixZmin, 4 FixInterior), stopping
 * when the mean step (end_if_small_step = 1, ConvCrit = Step) or the squared
 * gradient norm (0) falls to tol, or after max_iter iterations; the relaxed
 * displacements replace the context's (the build then uses them) and are
 * copied to dsp if it is not NULL; *energy at the result, *iterations. */
int tbgpu_vff_energy(tbgpu_ctx *ctx, const double *vff, double *energy, double *grad);
int tbgpu_vff_relax(tbgpu_ctx *ctx, const double *vff, int bc, int max_iter, double tol,
                    int end_if_small_step, double *energy, int *iterations, double *dsp);

/* Momentum (optical) matrix elements of n eigenstates psi_dev ([n][dimension]
 * complex, device) and their Kramers partners, for x, y and z: the
 * reference's MOMENTUM_MATRIX block (nemo3d/src/base/eigsys3d_par.c:410-640,
 * COMPUTE_Px/Py/Pz), p = i(<a|H r b> - <a|r H b>) with r the strained atom
 * coordinate (nm) and (a, b) = (psi_i, psi_f), (psi_i, psi'_f), (psi'_i,
 * psi_f), (psi'_i, psi'_f), psi' = (-conj(psi_down), conj(psi_up)).
 * P (host, or NULL): [3][n][8n] complex in the reference's pXmatrix layout,
 * entry [d][i][8f + 2c] = label (+-(i+1), +-(f+1)), a minus sign marking
 * the partner, [8f + 2c + 1] = p.  trans (host, or NULL; needs E, the n
 * eigenvalues): [3][n(n-1)/2][4] = (istate, fstate, E_i - E_f, sum of |p|^2
 * over the four pairs) for istate > fstate, fstate outer (TransProbX).
 * Spin models only, at the Gamma point (else TBGPU_E_UNSUPPORTED); 2n H*x
 * products and one fused pass over the vectors. */
int tbgpu_momentum_matrix(tbgpu_ctx *ctx, int n, const double *psi_dev, const double *E,
                          double *P, double *trans);

/* Timing of the last solve / build (ms, CUDA events on the context stream). */
/* ---- Learned warm start (no counterpart in the reference) -------------
 * A 3-D convolutional network on a G^3 grid over the structure's cells
 * predicts the in-gap shift sigma and K band-edge envelopes, which shape the
 * Lanczos start vector (the r_0 seam of tbgpu_eigensolve_lanczos, where the
 * reference uses rand() or a file).  These are its kernels; the network,
 * its training loop and the cold-start fallback are host code
 * (nemo3d_b200/warmstart.py).  Device pointers; activations float
 * [n][c][G^3] (voxel index (x*G + y)*G + z, cell i in voxel i*G/nx),
 * weights bf16 [cout][cin][27] (tap (dx+1)*9 + (dy+1)*3 + dz+1), float
 * accumulation; channels 1..32, G 1..64, else TBGPU_E_ARG.  The
 * context-free kernels run on the legacy default stream. */
/* features [3][G^3]: In fraction of the cation sites (species in_species),
 * site occupancy, mean displacement length (pm); synchronous */
int tbgpu_ws_features(tbgpu_ctx *ctx, int G, int in_species, float *feat_dev);
/* out = conv(in) + bias, ReLU on the output when relu != 0 */
int tbgpu_ws_conv3d_fwd(const float *in_dev, const uint16_t *w_dev, const float *bias_dev,
                        float *out_dev, int n, int cin, int cout, int G, int relu);
/* din = conv^T(g), g = dout masked by act > 0 (act = the layer's stored
 * ReLU output, or NULL for a linear layer) */
int tbgpu_ws_conv3d_bwd_data(const float *dout_dev, const float *act_dev, const uint16_t *w_dev,
                             float *din_dev, int n, int cin, int cout, int G);
/* dw [cout][cin][27] and db [cout] from the layer input and g as above */
int tbgpu_ws_conv3d_bwd_weight(const float *in_dev, const float *dout_dev, const float *act_dev,
                               float *dw_dev, float *db_dev, int n, int cin, int cout, int G);
/* out [n][k+1][G^3]: sigma_pred[n] = grid mean of channel k.  With targets
 * env [n][k][G^3] and sigma [n]: loss = mean (out - env)^2 over the first k
 * channels + w_sigma * mean_n (sigma_pred - sigma)^2, dout its gradient;
 * env = NULL computes sigma_pred alone */
int tbgpu_ws_loss(const float *out_dev, const float *env_dev, const float *sigma_dev, int n, int k,
                  int G, float w_sigma, float *dout_dev, float *sigma_pred_dev, float *loss_dev);
/* Adam step (bias-corrected, step >= 1) on float w; wbf = bf16(w) */
int tbgpu_ws_adam(float *w_dev, uint16_t *wbf_dev, const float *g_dev, float *m_dev,
                  float *v_dev, long n, float lr, float b1, float b2, float eps, int step);
/* r0[a][o] = u[a][o] * sqrt(sum_q env[q][voxel(a)]^2 prof[q][sub(a)][o] +
 * floor_w), sub = 0 for cation sites, 1 for anion sites; u and r0 complex
 * [dimension] (each part scaled); synchronous */
int tbgpu_ws_start_vector(tbgpu_ctx *ctx, const float *env_dev, const float *prof_dev, int k,
                          int G, float floor_w, const double *u_dev, double *r0_dev);

typedef struct {
  double build_ms;            /* topology + assembly                          */
  double solve_ms;            /* eigensolve_lanczos, first pass               */
  double vectors_ms;          /* second pass (eigenvectors)                   */
  double spmv_ms;             /* sum over H*x launches (when profiling on)    */
  long spmv_launches;
  long lanczos_iterations;
  long kernel_launches;       /* all kernels launched by the last solve       */
  double refine_ms;           /* double-precision refinement (mixed solve)    */
  long vec_segments;          /* eigenvector pass 1: segments regenerated     */
  long vec_mismatch;          /* ... whose last vector differed, bit for bit, */
                              /* from the first pass's checkpoint (0 expected) */
  double update_ms;           /* sum over the recurrence's update launches     */
                              /* (when profiling on)                           */
  double check_ms;            /* host time in the convergence tests            */
  double wait_ms;             /* host time waiting for the GPU's check batches */
} tbgpu_stats;
int tbgpu_set_profiling(tbgpu_ctx *ctx, int on);

/* Folded-spectrum operator F = factor * (H - shift2)(H - shift1) + offset,
 * the reference's matvect_mult2 (nemo3d/src/base/h_cvectr_mult.c:156-198,
 * whose constants 1.38, 1.58, -10, 0 are the defaults here): eigenvalues of H
 * nearest (shift1 + shift2) / 2 become the largest of F when factor < 0.
 * tbgpu_set_fold(ctx, 1, ...) makes the Lanczos solves
 * (tbgpu_eigensolve_lanczos(_dev)) run on F: two products and one combining
 * pass per step (which also reduces alpha), the windows and the returned
 * values are those of F (as with the reference's driver on matvect_mult2),
 * the eigenvectors come from the second run of the recurrence, and
 * tbgpu_get_fold_energies returns <v, H v> / <v, v> of each returned
 * eigenvector (the energies of H).  Double precision only (a mixed-precision
 * context returns TBGPU_E_UNSUPPORTED).  0 turns it off.  Each product reads
 * H once, so F costs two reads of H per application. */
int tbgpu_set_fold(tbgpu_ctx *ctx, int on, double shift1, double shift2, double factor,
                   double offset);
/* Drop-in for the reference's matvect_mult2 (h_cvectr_mult.c:156): the
 * matmul signature, y = F x over host vectors (argList[1] is ignored, as
 * there).  Failures through tbgpu_last_error(). */
void tbgpu_matvect_mult2(const int **argList, tbgpu_dcomplex *y, const tbgpu_dcomplex *x);
/* y = F x on device vectors (16-byte aligned, distinct); asynchronous. */
int tbgpu_hx_fold_dev(tbgpu_ctx *ctx, const double *x_dev, double *y_dev);
/* <v, H v> / <v, v> of the eigenvectors of the last folded solve; returns
 * their count (writes at most cap). */
int tbgpu_get_fold_energies(const tbgpu_ctx *ctx, int cap, double *energies);

/* Eigenvector pass of the Lanczos solves (no counterpart in the reference,
 * whose eigenvectorsLanczos reruns the whole recurrence from the start
 * vector, eigen/src/lanczos.c:1364-1689).  mode 0 (default) is that second
 * run.  mode 1: the first pass also saves the two Lanczos vectors that start
 * every segment of `segment` iterations (2 vectors per segment in device
 * memory), and the eigenvector pass regenerates `columns` segments at once:
 * one product reads each bond block once for all of them (10-orbital models
 * with a stored Hamiltonian at the Gamma point; columns 1..4 for the
 * mixed-precision solve, 1..2 for double vectors), with the three-term
 * update fused into the product.  Every product of both passes then uses the
 * lane-per-(atom, spin) kernel (H*x variant 5), or the pencil kernel when
 * variant 6 is set, whose columns compute exactly as a one-column launch: the regenerated vectors equal the first
 * pass's bit for bit (checked at every segment end, tbgpu_stats.vec_mismatch),
 * so the eigenvalues are those of mode 0 and the eigenvectors differ only by
 * the order of the accumulation.  Where the mode does not apply, or the
 * checkpoints do not fit in device memory, the solve uses mode 0. */
int tbgpu_set_eigenvector_pass(tbgpu_ctx *ctx, int mode, int columns, int segment);
int tbgpu_get_stats(const tbgpu_ctx *ctx, tbgpu_stats *out);

/* Failure-detection self-test: one warp waits, with the bounded poll loop
 * (at most polls, 1..2^24) that every device-side wait of the library uses,
 * on an mbarrier that is never completed.  Returns TBGPU_E_TIMEOUT when the
 * wait ran out and reported itself as designed; the context stays usable.
 * These synchronous entry points read the same status word (a kernel's wait
 * that ran out) after their stream drains, clear it and return its code:
 * tbgpu_eigensolve_lanczos(_dev), tbgpu_eigensolve_lanczos_batched,
 * tbgpu_eigensolve_blk_lanczos(_dev), tbgpu_momentum_matrix,
 * tbgpu_matvect_mult (through tbgpu_last_error), tbgpu_vff_energy,
 * tbgpu_vff_relax and tbgpu_build_hamiltonian.  The asynchronous device
 * entry points (tbgpu_hx_dev, tbgpu_hx_dev_f32, tbgpu_hx_block_dev,
 * tbgpu_matvect_mult_dev, tbgpu_hx_dot_noalloc) leave it for the next
 * synchronous call on the context. */
int tbgpu_selftest_bounded_wait(tbgpu_ctx *ctx, long polls);

int tbgpu_last_error(void);
const char *tbgpu_error_string(int code);

#ifdef __cplusplus
}
#endif
#endif
