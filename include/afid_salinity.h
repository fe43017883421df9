/*
 * afid_salinity.h — the multi-resolution salinity scalar of AFiD-MuRPhFi on the device (C ABI).
 *
 * The reference evolves salinity on a refined grid (MULTIRES = 1, FLAGSAL = 1 in bou.in) and
 * couples it to the flow every substep (src/flow_solver/TimeMarcher.F90:50-63, 95, 138-144):
 *   ExplicitSalinity / ImplicitSalinity / SolveImpEqnUpdate_Sal   src/salinity.F90:268-453
 *   AddSalBuoyancy (into the forcing along gAxis)                 src/salinity.F90:494-506
 *   InterpVelMgrd (coarse velocity -> refined grid)               src/multires/InterpVelMgrd.F90
 *   InterpSalMultigrid (refined salinity -> coarse buoyancy)      src/salinity.F90:455-492
 *   the refined-grid CFL number CFLmr that the dt rule uses       src/flow_solver/CalcMaxCFL.F90:48-68
 *   CalcSalStats / CalcDissipationSal (means.h5 profiles)         src/salinity.F90:508-667
 * The grid and stencil set-up (CreateMgrdGrid.F90, CreateMgrdStencil.F90 and the Hermite
 * stencils of multires/HermiteInterpolations.F90:26-164) runs on the host: afid_mgrd_create
 * builds the afid_sal_grid_t that afid_gpu_sal_create takes.  Once enabled on a context,
 * afid_gpu_timemarcher / afid_gpu_substep advance salinity with the flow.
 *
 * Not on this path: phase-field, moisture, IBM (solidr masks) and melt boundary conditions.
 * Batches and served jobs carry no salinity.
 *
 * Interpolation stencils are given per target point: target n reads the four source rows
 * start[n] .. start[n]+3 (0-based) with weights w[4n .. 4n+3].  Along y and z the rows wrap
 * periodically.  Along x they index a wall-extended column: rows -2 .. nsrc+1, where -1 and nsrc
 * are the ghost rows of the reference (InterpVelMgrd.F90:40-41 for coarse velocity gradients,
 * salinity.F90:471-480 for refined salinity) and -2, nsrc+1 are zero.
 */
#ifndef AFID_SALINITY_H
#define AFID_SALINITY_H

#include <stdint.h>

#include "afid_gpu.h"
#include "afid_host.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct afid_stencil {
  int n;                 /* target points                                               */
  const int *start;      /* [n] first source row (0-based; see above)                    */
  const double *w;       /* [4n] weights, w[4*t + a] for source start[t] + a             */
} afid_stencil_t;

/* Refined grid, physics and stencils (CreateMgrdGrid.F90, CreateMgrdStencil.F90). */
typedef struct afid_sal_grid {
  int nxmr, nymr, nzmr;          /* refined cells (NXMR NYMR NZMR)                               */
  double dxr, dyr, dzr;          /* nxmr/alx3, nymr/ylen, nzmr/zlen  (CreateMgrdGrid.F90:95-97)  */
  double pecs;                   /* solutal Peclet number ren*PraS  (ReadInputFile.F90:122)      */
  double bycs;                   /* salinity buoyancy prefactor     (ReadInputFile.F90:111-119)  */
  int active_s;                  /* 1 = AddSalBuoyancy along gAxis                              */
  int sfixs, sfixn;              /* fixed-S (1) / zero-flux (0) lower and upper plates            */
  const double *xcr;             /* [nxmr+1] refined faces   CreateMgrdGrid.F90:50-90              */
  const double *udx3mr;          /* [nxmr]   dxr/d3xcr       CreateMgrdGrid.F90:130-133            */
  const double *g3rmr;           /* [nxmr]   centre metric   CreateMgrdGrid.F90:118-123            */
  const double *ap3sskr, *ac3sskr, *am3sskr; /* [nxmr] d2/dx2 with the SfixS/N ghosts        */
  const double *salbp, *saltp;   /* [nymr*nzmr] plate salinity, y fastest (SetSalBCs)           */
  afid_stencil_t to_ref[3];      /* coarse cell centres -> refined cell centres: x, y, z        */
  afid_stencil_t to_coarse[3];   /* refined salinity -> the salc points: x, y, z                 */
} afid_sal_grid_t;

/* ---- host set-up --------------------------------------------------------------------------- */
typedef struct afid_mgrd afid_mgrd_t;
/* CreateMgrdGrid + CreateMgrdStencil + SetSalBCs for the bou.in behind `coarse` (MULTIRES = 1,
 * FLAGSAL = 1, ISTR3R in {0, 1, 3, 4, 6, 7}, NZMR = 1 exactly when NZM = 1). */
int afid_mgrd_create(const afid_tables_t *coarse, afid_mgrd_t **out);
void afid_mgrd_destroy(afid_mgrd_t *m);
const afid_sal_grid_t *afid_mgrd_view(const afid_mgrd_t *m);
/* 1 when InterpSalMultigrid takes interpolate_xyz_to_coarse_fast (salinity.F90:485). */
int afid_mgrd_fast(const afid_mgrd_t *m);
/* named 1-D table ("xcr", "xmr", "g3rmr", "udx3mr", "ap3sskr", "ac3sskr", "am3sskr",
 * "cxrs", "cyrs", "czrs" ...); NULL if unknown; *len set */
const double *afid_mgrd_array(const afid_mgrd_t *m, const char *name, int *len);
/* CreateInitialSalinity (salinity.F90:140-170, non-IBM branches): the double-diffusive profile
 * 0.5 (2 (xmr - 0.5))^7 when active_S = active_T = 1 and gAxis = 1, else the linear profile plus
 * noise of amplitude amp limited to |S| <= 0.5, U from Philox keyed by k + (nxmr+1)(j + nymr i).
 * Fortran layout with leading dims ld_x >= nxmr, ld_y >= nymr. */
int afid_initial_salinity(const afid_mgrd_t *m, uint64_t seed, double amp, double *sal, int ld_x,
                          int ld_y);

/* ---- device ---------------------------------------------------------------------------------- */
#define AFID_NUM_SAL_PROFILES 6
/* Allocate the refined fields on a single-domain context and upload the tables.  Salinity starts
 * at zero; the flow's explicit terms take the salinity buoyancy from here on. */
int afid_gpu_sal_create(afid_ctx_t *ctx, const afid_sal_grid_t *sg);
/* Salinity from host (Fortran layout, ld_x >= nxmr, ld_y >= nymr), rusal zeroed, then the
 * initial InterpVelMgrd + InterpSalMultigrid of main.F90:206-208. */
int afid_gpu_sal_upload(afid_ctx_t *ctx, const double *sal, int ld_x, int ld_y);
int afid_gpu_sal_download(afid_ctx_t *ctx, double *sal, int ld_x, int ld_y);
/* InterpVelMgrd + InterpSalMultigrid from the resident state (after afid_gpu_upload). */
int afid_gpu_sal_interpolate(afid_ctx_t *ctx);
/* CFLmr (CalcMaxCFL.F90:48-65), at least 1e-8: the CFL number the dt rule uses with salinity. */
int afid_gpu_sal_cfl(afid_ctx_t *ctx, double *cflmr);
/* out[AFID_NUM_SAL_PROFILES * nxmr]: Sbar, Srms, vxS, vyS, vzS, chiS (CalcSalStats). */
int afid_gpu_sal_profiles(afid_ctx_t *ctx, double *out);
/* Plane mean of the refined salinity over y (axis 1: out[nzmr][nxmr], ymeanr of
 * h5tools/means.F90:84-157 without IBM) or over z (axis 2: out[nymr][nxmr], zmeanr). */
int afid_gpu_sal_mean_plane(afid_ctx_t *ctx, int axis, double *out);
/* The interpolated fields: vxr [nxmr+1 rows], vyr, vzr [nxmr rows] with leading dims
 * ldr_x >= nxmr+1, ldr_y >= nymr; salc [nxm rows] with ldc_x >= nxm, ldc_y >= nym.  NULL skips. */
int afid_gpu_sal_download_aux(afid_ctx_t *ctx, double *vxr, double *vyr, double *vzr, int ldr_x,
                              int ldr_y, double *salc, int ldc_x, int ldc_y);

#ifdef __cplusplus
}
#endif
#endif /* AFID_SALINITY_H */
