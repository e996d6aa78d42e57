/*
 * cgd_oracle.h - C interface of the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  This is an FP64 CPU restatement of the
 * reference's spectral-element hot path (CGDycore.jl), used by the test suite,
 * by __graft_entry__.smoke() and by bench.py's CPU-baseline leg as the
 * checker.  The product library (libcgd_b200.so) never links or calls it.
 *
 * Arrays follow the reference's column-major (Julia) layouts:
 *   Glob   (N*N, NF)            int64, 1-based
 *   X      (N*N, 2, 3, nz, NF)  node coordinates at the bottom/top of a layer
 *   dXdxI  (3, 3, 2, N*N, nz, NF)
 *   J      (N*N, 2, nz, NF)
 *   M      (nz, NumG, 2)   MMass (nz, NumG)   dz (nz, NumG)
 *   U, F   (nz, NumG, NV)  NV = 5 + NumTr : rho, u, v, w, rho*theta, rho*q...
 */
#ifndef CGD_ORACLE_H
#define CGD_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_cfg {
  int nPanel;      /* cubed-sphere elements per panel edge */
  int OrdPoly;     /* polynomial order p (N = p+1 GLL nodes) */
  int nz;          /* vertical layers */
  int NumTr;       /* passive tracers */
  double Rad;      /* sphere radius = Phys.RadEarth */
  double H;        /* model top (Sleve reference height) */
  double HyperDCurl, HyperDGrad, HyperDDiv;
  double Up;       /* baroclinic-wave zonal-wind bump amplitude */
} orc_cfg;

void *orc_create(const orc_cfg *cfg, const double *zlev /* nz+1 */);
void orc_destroy(void *h);
int orc_set_threads(int n);
/* out: NF, NumG, DoF, N, NumNodes, NumEdges */
int orc_sizes(void *h, int64_t *out);
int orc_get_glob(void *h, int64_t *glob1);
int orc_get_gll(void *h, double *xw, double *w, double *DS, double *DW);
int orc_get_faces(void *h, double *F /* (4,3,NF) */);
int orc_get_metric(void *h, double *X, double *dXdxI, double *J);
int orc_get_mass(void *h, double *M, double *MMass);
int orc_get_dz(void *h, double *dz);
/* Replace the metric/mass/dz the oracle uses (e.g. arrays built elsewhere). */
int orc_set_metric(void *h, const double *X, const double *dXdxI, const double *J,
                   const double *M, const double *dz);
/* Baroclinic-wave state; tracer blob centres (lon,lat) pairs, NumTr of them. */
int orc_init_state(void *h, double *U, const double *tracer_lonlat);
int orc_pressure(void *h, const double *U, double *p);
/* Phase-1 hyperviscosity + DSS (Temp1 (nz,NumG,5+NumTr)). */
int orc_hypervisc1(void *h, const double *U, double *Temp1);
/* Full tendency FcnPrepare + Fcn (F (nz,NumG,NV)). */
int orc_rhs(void *h, const double *U, double *F);
/* Jacobian bands JRhoW, JWRho, JWRhoTh, JRhoThW, each (2, nz-1, NumG). */
int orc_jac(void *h, const double *U, double *bands);
/* Schur column solve: k (nz,NumG,NV) from v (modified) with fac = dt*gamma,
 * using the bands of the last orc_jac call. */
int orc_schur(void *h, double *k, double *v, double fac);
/* nsteps SSP-Knoth Rosenbrock-W steps in place. */
int orc_ros_step(void *h, double *U, double dt, int nsteps);
/* sum(rho * MMass) */
double orc_mass_integral(void *h, const double *U);

/* Output interpolation to OrdPrint x OrdPrint sub-cells (src/Outputs):
 * inter (OrdPrint, OrdPrint, N, N), cell (OrdPrint, OrdPrint, nz, NF).
 * kind 0: c (divided by rhoc when not NULL), 1: dry pressure of c = rho*theta,
 * 2: dry potential temperature of c = rho*theta and rhoc = rho. */
int orc_vtk_inter(int OrdPoly, int OrdPrint, const double *xw, double *inter);
int orc_interpolate(void *h, const double *c, const double *rhoc, int kind, const double *inter, int OrdPrint,
                    double *cell);
int orc_interpolate_wb(void *h, const double *u, const double *v, const double *w, const double *inter,
                       int OrdPrint, double *cell);
int orc_interpolate_vort(void *h, const double *U, const double *inter, int OrdPrint, double *cell);

#ifdef __cplusplus
}
#endif
#endif
