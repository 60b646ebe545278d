/* CPU oracle for the scadyn T-matrix solve path — TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of the reference's Fortran algorithm (jherrane/scadyn,
 * src/ Fortran files), used only by tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg, to check results.  Nothing in the product links or calls it.
 *
 * Parity status: UNPINNED by the reference's own tests — the reference ships
 * no tests, golden vectors or fixtures, and cannot be compiled here (no
 * Fortran compiler, FFTW, LAPACK or HDF5).  The restatement is cross-checked
 * against an independent numpy/scipy restatement (tests/) and against the
 * Mie series for spheres (src/mie.f90:99-172).
 *
 * Array conventions follow the reference (Fortran column-major, 1-based ids):
 *   coord  (3,Nv) double          -> coord[3*v + d]
 *   etopol (4,T)  int32, 1-based  -> etopol[4*t + c]
 *   S      (27,T) complex double  -> S[27*t + j]
 *   indS   (27,T) int32, 1-based grid node ids
 *   sp_mat (3,3,B) complex float  -> sp_mat[9*b + r + 3*c]
 *   sp_ind (2,B)  int32, 1-based tet ids (tet_T, tet_B)
 *   Fg     (2Nx,2Ny,2Nz) complex double, x fastest
 */
#ifndef SCADYN_ORACLE_H
#define SCADYN_ORACLE_H
#include <stdint.h>
#include <complex.h>
#include <stddef.h>

typedef double _Complex zc;
typedef float _Complex  fc;

typedef struct {
    /* mesh (borrowed) */
    int Nv, T;
    const double *coord;
    const int32_t *etopol;
    const zc *param;
    /* parameters (src/common.f90:78-89 defaults) */
    double grid_size;   /* "cell_size" */
    int M_ex;           /* 2 */
    int near_zone;      /* 1 */
    double k;
    /* build_grid / build_box / tetras_in_cubes outputs */
    int Nx, Ny, Nz;
    double delta, box_delta, min_coord[3];
    int Nx_cube, Ny_cube, Nz_cube, N_cubes;
    int32_t *etopol_box;    /* (27, N_cubes) 1-based node ids */
    int N_tet_cube;
    int32_t *tetras;        /* (N_tet_cube, N_cubes) 1-based tet ids, 0 = none */
} orc_geom;

#ifdef __cplusplus
extern "C" {
#endif

/* geometry (src/geometry.f90) */
int  orc_geom_build(orc_geom *g);                 /* build_grid + build_box + tetras_in_cubes */
void orc_geom_free(orc_geom *g);
int  orc_find_near_cubes(const orc_geom *g, int cube, int32_t *out); /* (2nz+1)^3 entries */
int  orc_point_in_cube(const orc_geom *g, const double p[3]);
void orc_node_coord(const orc_geom *g, int node1, double out[3]);

/* projectors (src/projection.f90:17-166) */
int  orc_pfft_projection_const(const orc_geom *g, zc *S, zc *Sx, zc *Sy, zc *Sz, int32_t *indS);
int  orc_pinv(int M, int N, const zc *A, zc *Ainv);   /* (M,N) -> (N,M), cut s > 1e-6 */

/* near zone (src/precorrection.f90:131-264) */
int64_t orc_nearzone_count(const orc_geom *g);
int  orc_nearzone_const(const orc_geom *g, const zc *S, const zc *Sx, const zc *Sy, const zc *Sz,
                        int64_t B, fc *sp_mat32, zc *sp_mat64, int32_t *sp_ind, int nthreads);

/* linear basis set-up (mesh%order = 1): projectors (27, 4T) with column
 * 4(t-1)+n for node n of tet t (src/projection.f90:170-338), and 12x12 near-zone
 * blocks sp(12,12,B) over the same tet pairs as the constant basis
 * (src/precorrection.f90:268-725, src/singularity_subtraction_N.f90) */
int  orc_pfft_projection_lin(const orc_geom *g, zc *S, zc *Sx, zc *Sy, zc *Sz, int32_t *indS);
int  orc_nearzone_lin(const orc_geom *g, const zc *S, const zc *Sx, const zc *Sy, const zc *Sz,
                      int64_t B, fc *sp_mat32, zc *sp_mat64, int32_t *sp_ind, int nthreads);

/* test forms: singularity_subtraction_int_V_GN / _int_S_GN at one point with
 * the order-5 rules, B (4,3) and tri (3,3) vertex coordinates; gradshape */
void orc_int_V_GN(const double rf[3], double k, const double B[12], zc out[4]);
void orc_analytical_integration(const double tri[9], const double r[3], double out[2]);  /* int 1/R, int R */
zc   orc_int_V_G(const double rf[3], double k, const double B[12]);
zc   orc_int_S_G(const double rf[3], double k, const double tri[9]);
void orc_int_S_GN(const double rf[3], const double tri[9], double k, zc out[3]);
void orc_gradshape(const double tc[12], double dN[12]);

/* Green's function grid (src/build_G.f90) */
int  orc_build_G(const orc_geom *g, zc *Fg);

/* 1D/3D FFT helpers (FFTW semantics: forward exp(-i), unnormalised) */
int  orc_fft1d(int L, zc *x, int sign);
int  orc_fft3d(int Px, int Py, int Pz, zc *A, int sign);
int  orc_fft3d_pruned(int Px, int Py, int Pz, zc *A, int inverse);

/* matvec pieces (src/sparse.f90, src/sparse_mat.f90, src/gmres_module.f90) */
void orc_sparse_T_matmul(int T, const zc *val, const int32_t *ind, const zc *x, int Ngrid, zc *out);
void orc_sparse_eps_matmul(int T, const zc *val, const int32_t *ind, const zc *x, zc *out);
void orc_matmul_Acorr_const(int T, int64_t B, const fc *sp32, const zc *sp64, const int32_t *sp_ind,
                            const zc *x, zc *Ax, int nthreads);

typedef struct {
    const orc_geom *g;
    int T;
    const zc *S, *Sx, *Sy, *Sz;
    const int32_t *indS;
    const zc *Fg;              /* (2Nx,2Ny,2Nz) */
    int64_t B;
    const fc *sp32;            /* faithful complex64 storage, or NULL */
    const zc *sp64;            /* FP64 storage, or NULL */
    const int32_t *sp_ind;
    double k;
    int merged;                /* 0: six convolutions as the reference; 1: four */
    int nthreads;
    int order;                 /* basis order: 0 constant (3 unknowns per tet), 1 linear (12: 4 nodes x 3) */
} orc_op;

int  orc_compute_Ax2(const orc_op *op, const zc *x, zc *Ax);
/* matmul_Acorr (src/sparse_mat.f90:64-92): 12x12 blocks of the linear basis */
void orc_matmul_Acorr(int T, int64_t B, const fc *sp32, const zc *sp64, const int32_t *sp_ind,
                      const zc *x, zc *Ax);

/* restarted GMRES (src/gmres_module.f90:180-325) */
typedef struct {
    int iters;           /* Arnoldi steps taken */
    int matvecs;         /* operator applications */
    int cycles;
    int converged;
    double relres;       /* |g(i+1)|/||b|| at exit */
    double *history;     /* optional, length >= m*cycles */
    int history_len;
} orc_gmres_info;
int  orc_gmres(const orc_op *op, const zc *rhs, zc *x, double tol, int m, int cycles,
               orc_gmres_info *info);
void orc_mgs_terms(size_t n, int i, const zc *V, zc *w, zc *h);   /* one Arnoldi step's MGS over i vectors */

/* incident VSWFs and T assembly (src/T_matrix.f90:240-305, src/mie.f90:408-496) */
int  orc_calc_MN(int Nmax, zc k, const double Po[3], zc *MM, zc *NN);   /* (3,nm) each */
int  orc_vswf2constant(const double *coord, const int32_t *etopol, int T, zc k, int Nmax, zc *mat);
void orc_cspherebessel(int n, zc z, zc *csj, zc *csy);                    /* 0..n */
void orc_legendre2(int N, double x, double *P);                            /* N+1 */
void orc_T_assemble(int n, int ncol, const zc *mat, const zc *X, zc *Tcols);/* matᴴX */
int  orc_mie_T(int Nmax, double ka, zc m, zc *a_n, zc *b_n);               /* a_n, b_n */
void orc_tr_T(int nm, const zc *Taa, const zc *Tbb, const zc *Tab, const zc *Tba, double k, double crs[4]);

#ifdef __cplusplus
}
#endif
#endif
