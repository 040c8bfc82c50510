/*
 * tb_oracle.h -- CPU oracle for the tight-binding eigensolver hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of NEMO-3D's
 * Hamiltonian assembly, H*x and Lanczos driver, used by the test-suite and by
 * the CPU-baseline leg of bench.py as the checker.  The product (libtbgpu.so)
 * never links, loads or calls it.
 *
 * Every function cites the reference routine it restates.  Paths are relative
 * to the NEMO-3D source tree.
 */
#ifndef TB_ORACLE_H
#define TB_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NPV 35   /* sp3d5s* parameter vector length (mb_ham_spds_micro.h:82) */
#define ORC_NSTR 33  /* strain vector length (mb_ham_spds_micro.h:87) */
#define ORC_NPAR (ORC_NPV + ORC_NSTR)

typedef struct {
  int nx, ny, nz;             /* dense cell grid, cell (i,j,k) row-major, k fastest */
  int periodic[3];            /* 1 = periodic along that axis                    */
  double lattice[3];          /* device lattice constants a_x, a_y, a_z (nm)      */
  const unsigned char *type;  /* [nx*ny*nz*8] species id per site, 0 = empty      */
  const double *dsp;          /* [nx*ny*nz*8*3] displacements (nm) or NULL       */
} orc_geom;

typedef struct {
  int norb;                   /* orbitals per spin: 5 (sp3s*) or 10 (sp3d5s*)     */
  int nspin;                  /* 1 or 2                                           */
  int include_strain;         /* ElCalc.include_strain_in_Hamiltonian             */
  int passivate;              /* SurfacePassivation == PassivateDanglingBond      */
  double dangling_shift;      /* Phys.DanglingBondEnergyShift (eV)                */
  int nspecies;               /* species ids are 0..nspecies-1                   */
  const double *par;          /* [nspecies][nspecies][ORC_NPAR] prepared (c,a)    */
  const unsigned char *par_ok;/* [nspecies][nspecies] 1 where a set exists        */
} orc_model;

/* param_init for one material: returns 0, fills out[ORC_NPAR]. */
int orc_prepare_params(int sp3s_family, int include_strain, const double *mb_pv,
                       const double *mb_strain, double ev_offset, double a0,
                       double *out);

/* Zincblende topology.  Returns the number of atoms (or -1 if max_atoms is too
 * small).  atom_slot[a] = site index; nbr[a*4+n] = neighbour atom or -1;
 * wrap[(a*4+n)*3+d] = -1/0/+1 periodic image crossed; surface[a] = 1 if the
 * atom has fewer than 4 neighbours. */
long orc_topology(const orc_geom *g, long max_atoms, int *atom_slot, int *nbr,
                  signed char *wrap, unsigned char *surface);

/* Assemble the stored Hamiltonian.  onsite: [natoms][nb][nb] complex (re,im)
 * with nb = norb*nspin; blocks: [natoms][4][norb][norb] real, filled for cation
 * atoms only, block[c][a] = <anion orbital a | H | cation orbital c>.
 * Returns 0, or a negative code on a missing material set. */
int orc_build(const orc_geom *g, const orc_model *m, long natoms,
              const int *atom_slot, const int *nbr, const signed char *wrap,
              const unsigned char *surface, double *onsite, double *blocks);

/* Building blocks of orc_build, exposed for checks against the reference's
 * own routines.  orc_onsite_block: h3d_diag for one atom (h [nb][nb]
 * complex).  orc_bond: one bond seen from "this" atom, nnv and nnv0 pointing
 * anion -> cation; blk[c][a] = <anion a|H|cation c>; the strain correction of
 * this atom's on-site energies is added to ediag[norb]. */
void orc_onsite_block(int norb, int nspin, int cation, const double *p, double *h);
void orc_bond(int norb, int this_cation, const double *nnv, const double *nnv0,
              const double *par, int use_strain, double a0, double *blk,
              double *ediag);

/* y = (H - shift) x with per-bond Bloch phases k (NULL = Gamma / closed).
 * x,y: [natoms][nb] complex interleaved. */
void orc_hx(int norb, int nspin, long natoms, const int *atom_slot,
            const int *nbr, const signed char *wrap, const double *kvec, const double *onsite,
            const double *blocks, double shift, const double *x, double *y);

/* Dense Hermitian H(k) (n x n complex, row-major) for small systems. */
void orc_dense(int norb, int nspin, long natoms, const int *atom_slot,
               const int *nbr, const signed char *wrap, const double *kvec, const double *onsite,
               const double *blocks, double *h);

/* Eigenvalues of a real symmetric tridiagonal matrix in (vl, vu], ascending
 * (restates the use of LAPACK dstebz RANGE='V' ORDER='E' in lanczos.c:793-811). */
int orc_tridiag_eigs(int n, const double *diag, const double *offd, double vl,
                     double vu, double abstol, double *w);

typedef void (*orc_matvec_fn)(void *ctx, const double *x, double *y);

typedef struct {
  int conv_start, conv_skip, imax;   /* ConvCheckStartIter, SkipRate, MaxIter */
  int req1, req2;                    /* NumEigReq_vb, NumEigReq_cb            */
  double emin1, emax1, emin2, emax2; /* Erange_vb, Erange_cb                  */
  double tolerance;                  /* ConvTolerance                         */
  unsigned int seed;                 /* seed of the inverse-iteration starts  */
} orc_lanczos_opts;

/* eigensolve_lanczos (lanczos.c:1823-2089): returns the number of eigenvalues
 * found; evals[nfound] ascending; conv_it[nfound]; *iterations;
 * if evecs != NULL, evecs[nfound][n] complex from the second Lanczos pass.
 * alpha/beta (length >= imax) receive the tridiagonal matrix. */
int orc_eigensolve_lanczos(orc_matvec_fn mv, void *ctx, long n, const double *r0,
                           const orc_lanczos_opts *o, double *evals,
                           int *conv_it, int *iterations, double *evecs,
                           double *alpha, double *beta);

/* Matvec context over an assembled oracle Hamiltonian. */
typedef struct {
  int norb, nspin;
  long natoms;
  const int *atom_slot;
  const int *nbr;
  const signed char *wrap;
  const double *kvec;
  const double *onsite;
  const double *blocks;
  double shift;
} orc_ham;
void orc_ham_matvec(void *ham, const double *x, double *y);

/* Keating VFF energy (StrainModel = VFF_keating, calc_estrain,
 * base/strain3d.c:1361-2080) at displacements u[natoms*3] (nm, atom order);
 * grad[natoms*3] = dE/du.  vff: [ns][ns][3] = (a0 nm, alpha, beta) per
 * species pair. */
double orc_vff_energy(const orc_geom *g, long natoms, const int *atom_slot, const int *nbr,
                      int ns, const double *vff, const double *u, double *grad);
/* Free atoms under boundary condition bc (0 AllFree, 1 FixOne,
 * 2 FixSurfaceAll, 3 FixZmin, 4 FixInterior). */
void orc_vff_free_mask(const orc_geom *g, long natoms, const int *atom_slot,
                       const unsigned char *surface, int bc, unsigned char *free_mask);
/* min_estrain with macoptII_par (eigen/src/macopt_par.c:121-475): u is
 * relaxed in place; returns the iteration count, *energy at the result. */
int orc_vff_relax(const orc_geom *g, long natoms, const int *atom_slot, const int *nbr,
                  const unsigned char *surface, int ns, const double *vff, int bc, int itmax,
                  double tol, int end_if_small_step, double *u, double *energy);

/* Host threads of the oracle's OpenMP loops. */
void orc_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
