/*
 * afid_continua.h — restart files in the reference's HDF5 layout (C ABI, plain C types).
 *
 * The reference writes one file per field through the HDF5 library and a master file with the
 * grid description; a run with NREAD = 1 reads them back.  These entry points produce and read
 * the same files without the HDF5 library:
 *
 *   afid_write_flow_field        WriteFlowField.F90:11-86: <dir>/continua_{temp,vx,vy,vz,[sal],pr}.h5
 *                                and <dir>/continua_master.h5 when final, otherwise
 *                                <dir>/fields/NNNNN_{temp,vx,vy,vz,[sal]}.h5 with
 *                                NNNNN = nint(time / save_3d)
 *   afid_read_continua_master    ReadFlowInterp.F90:23-58 (the master datasets)
 *   afid_read_flow_field         ReadFlowInterp.F90:76-171, same-grid branch: domain-size check,
 *                                grid check, then HdfReadContinua (h5tools/HdfReadContinua.F90) per
 *                                field; continua_pr.h5 is read only when it exists
 *   afid_read_flow_interp        ReadFlowInterp.F90 with both branches: on another grid the fields are
 *                                interpolated (InterpInputVel.F90, InterpInputSal.F90)
 *   afid_gpu_write_flow_field /  the same through a device context: download, write / read,
 *   afid_gpu_read_flow_field     upload (salinity included when the context has it)
 *   afid_write_grid_info         the coordinates file cordin_info.h5 (WriteGridInfo.F90)
 *   afid_write_means             the mean-profile file means.h5 (CalcMeanProfiles.F90:209-334)
 *   afid_write_movie             the movie-plane files flowmov/movie_{x,y,z}cut.h5 (MakeMovie*Cut.F90)
 *   afid_write_movie_mean        the plane-mean files flowmov/movie_{y,z}mean.h5 (mean_zplane.F90)
 *   afid_write_spectrum /        the spectrum files {vx,vy,vz,te}_spectrum.h5 (spectra.F90:169-196)
 *   afid_gpu_write_spectra
 *   afid_run_io                  afid_run plus the main loop's restart and save points:
 *                                ReadFlowInterp (either branch) when NREAD = 1 (main.F90:157-161), the start-up
 *                                frame (main.F90:241), the SAVE_3D frames (main.F90:376-381) and
 *                                the final continua files on a normal exit (QuitRoutine.F90:37)
 *
 * Each field file holds one dataset "var" of little-endian IEEE doubles with C-order dims
 * (nzm, nym, nx) — Fortran (nx, nym, nzm), h5tools/HdfRoutines.F90:467-471 — contiguous
 * storage; the refined salinity file has (nzmr, nymr, nxmr + 1) (HdfRoutines.F90:562-566).
 * The master file holds one-element datasets: nx, ny, nz, istr3 (32-bit integers), ylen, zlen,
 * time, str3 (doubles), and nxr, nyr, nzr, istr3r when MULTIRES = 1 (WriteFlowField.F90:54-81).
 * nx, ny, nz are nxm + 1, nym + 1, nzm + 1 as in param.F90; nxr, nyr, nzr likewise refined.
 *
 * Host arrays here are packed: vx, vy, vz, temp, pr with x extent nx (index nx - 1 is the upper
 * wall node, zero for the cell-centred fields), salinity with x extent nxmr.  The salinity file's
 * extra x node (nxmr + 1) is written as zero and dropped on reading.
 *
 * The container (afid_h5_*) is the subset of the HDF5 file format these files need: superblock
 * version 0, version-1 object headers, symbol-table groups (nested, any number of members),
 * fixed-point and floating-point datasets with contiguous storage.  The reader also takes superblock versions 1-3, version-2
 * object headers, compact link-message groups and compact storage; chunked storage, filters and
 * dense link storage are refused with AFID_E_IO.
 */
#ifndef AFID_CONTINUA_H
#define AFID_CONTINUA_H

#include <stdint.h>

#include "afid_gpu.h"
#include "afid_host.h"
#include "afid_salinity.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- the container ------------------------------------------------------------------------ */
#define AFID_H5_F64 1          /* IEEE binary64, little-endian on disk                       */
#define AFID_H5_I32 2          /* two's-complement 32-bit, little-endian on disk              */
#define AFID_H5_GROUP 3        /* an entry that only creates the (possibly empty) group `name` */
#define AFID_H5_MAX_RANK 4

typedef struct afid_h5_dataset {
  const char *name;            /* path below the root group: components of at most 255 bytes
                                  separated by '/'; the groups on the way are created         */
  int dtype;                   /* AFID_H5_F64 / AFID_H5_I32, or AFID_H5_GROUP (rank, dims and
                                  data ignored)                                               */
  int rank;                    /* 1 .. AFID_H5_MAX_RANK                                        */
  int64_t dims[AFID_H5_MAX_RANK];   /* C order: dims[rank - 1] varies fastest                  */
  const void *data;            /* prod(dims) host values of the type                           */
} afid_h5_dataset_t;

/* Create (truncate) path holding the n datasets (and groups).  Groups are symbol-table groups
 * whose B-trees grow extra levels as needed (more than 256 members per group are fine). */
int afid_h5_write(const char *path, int n, const afid_h5_dataset_t *sets);
/* Class and shape of one dataset: *dtype is AFID_H5_F64 for any floating-point type and
 * AFID_H5_I32 for any integer type.  AFID_E_IO if the file or dataset is missing or unsupported. */
int afid_h5_info(const char *path, const char *name, int *dtype, int *rank, int64_t dims[AFID_H5_MAX_RANK]);
/* Read a whole dataset converted to double (count must equal its element count). */
int afid_h5_read_f64(const char *path, const char *name, double *out, int64_t count);

/* ---- continua files ----------------------------------------------------------------------- */
typedef struct afid_continua_master {
  int nx, ny, nz;              /* nxm + 1, nym + 1, nzm + 1                                    */
  double ylen, zlen, time;
  int istr3;
  double str3;
  int multires;                /* 1: nxr, nyr, nzr, istr3r are written / read                 */
  int nxr, nyr, nzr, istr3r;   /* nxmr + 1, nymr + 1, nzmr + 1, ISTR3R                        */
} afid_continua_master_t;

/* The master record of a run described by in at the given time. */
int afid_continua_master_from_input(const afid_input_t *in, double time, afid_continua_master_t *m);
/* final != 0: continua_*.h5 including pr, and continua_master.h5; final == 0: a fields/ frame
 * without pr (pr may be NULL then).  sal is written when m->multires and sal != NULL.
 * Missing directories (dir, dir/fields) are created. */
int afid_write_flow_field(const char *dir, int final, double save_3d, const afid_continua_master_t *m,
                          const double *vx, const double *vy, const double *vz, const double *temp,
                          const double *pr, const double *sal);
/* Reads nx, ny, nz, time, istr3, str3, ylen, zlen, and the refined sizes when multires != 0. */
int afid_read_continua_master(const char *dir, int multires, afid_continua_master_t *m);
/* Same-grid restart into the current grid described by cur (time ignored): AFID_E_INVALID when
 * |ylen - ylen_old| or |zlen - zlen_old| > 1e-8, or when any size, istr3, str3 (1e-8) or refined
 * size differs (afid_read_flow_interp takes the interpolating branch then).  Fields are read
 * into the packed host arrays; pr only when continua_pr.h5 exists (*pr_read = 1), salinity when
 * cur->multires and sal != NULL.  *time_out gets the master's time. */
int afid_read_flow_field(const char *dir, const afid_continua_master_t *cur, double *time_out, double *vx,
                         double *vy, double *vz, double *temp, double *pr, int *pr_read, double *sal);

/* ReadFlowInterp.F90 as a whole for the run described by in: the same-grid branch above when
 * the stored grid matches (*interpolated = 0), otherwise the interpolating branch
 * (ReadFlowInterp.F90:85-136, *interpolated = 1): the old grid rebuilt from the master record
 * (CreateOldGrid.F90), cell-centre Hermite stencils old -> new (CreateNewInputStencil.F90),
 * velocities rebuilt from their interpolated gradients and temperature interpolated with the plate
 * ghosts (InterpInputVel.F90), the refined salinity interpolated likewise (InterpInputSal.F90);
 * the pressure is set to zero (*pr_read = 0).  Ly/Lz must match as in the same-grid branch, and a
 * 2-D file restarts a 2-D run only. */
int afid_read_flow_interp(const char *dir, const afid_input_t *in, double *time_out, double *vx, double *vy,
                          double *vz, double *temp, double *pr, int *pr_read, int *interpolated, double *sal);

/* ---- mean profiles file ------------------------------------------------------------------ */
/* <dir>/means.h5 as CalcMeanProfiles.F90:209-270 (HdfCreateMeansFile :289-334) and
 * CalcSalStats / CreateSalinityH5Groups (salinity.F90:592-603, :704-714) lay it out: one group per
 * profile (Tbar, vybar, vzbar, vxT, vyT, vzT, Trms, vxrms, vyrms, vzrms, vxvy, vxvz, vyvz, chiT,
 * epsilon; with salinity also Sbar, Srms, vxS, vyS, vzS, chiS), holding one dataset of nxm (nxmr)
 * doubles per sample, named NNNNN = nint(time / TOUT).  profiles[s][q][k] is sample s as
 * afid_gpu_mean_profiles returns it; sal_profiles[s][q][k] as afid_gpu_sal_profiles (NULL: no
 * salinity groups).  The reference appends each sample to the file as it is taken; this call
 * writes the whole file from the samples given (nsamples = 0: the empty groups).  Two samples
 * with the same NNNNN are refused (AFID_E_INVALID), as the reference cannot create a dataset twice. */
int afid_write_means(const char *dir, double tout, int nsamples, const double *times, int nxm,
                     const double *profiles, int nxmr, const double *sal_profiles);

/* ---- grid coordinates --------------------------------------------------------------------- */
/* <dir>/cordin_info.h5 as WriteGridInfo.F90:20-45 writes it: xm (nxm), xc (nx), ym (nym), zm
 * (nzm) of the grid in t and, when m is given (MULTIRES), xmr (nxmr), xcr (nxmr + 1), ymr (nymr),
 * zmr (nzmr) of the refined grid; the post-processing reads the coordinates from here. */
int afid_write_grid_info(const char *dir, const afid_tables_t *t, const afid_mgrd_t *m);

/* ---- movie planes ------------------------------------------------------------------------ */
/* <dir>/flowmov/movie_{x,y,z}cut.h5 (axis 0, 1, 2) as h5tools/MakeMovie{X,Y,Z}Cut.F90 and
 * h5tools/h5_tools.F90:33-135 lay them out: groups vx, vy, vz, temp (and sal), one 2-D dataset
 * per frame named NNNNN = nint(time / TFRAME).  planes[f][4][...] holds, per frame, the four planes
 * in afid_gpu_slice's layout for the axis (x: nzm x nym; y: nzm x nx; z: nym x nx; the y and z
 * cuts of vy, vz, temp are stored with their nxm cell rows, as the reference writes them);
 * sal_planes[f][...] the refined salinity planes (x: nzmr x nymr; y: nzmr x nxmr; z: nymr x nxmr)
 * or NULL.  The reference cuts at x index 1 (vx: 2), y index nym/2 + 1 and z index nzm/2 + 1
 * (1-based).  A later frame with the same number replaces an earlier one, as the reference
 * deletes and rewrites an existing dataset.  The whole file is written from the frames given. */
int afid_write_movie(const char *dir, int axis, double tframe, int nframes, const double *times, int nxm,
                     int nym, int nzm, const double *planes, int nxmr, int nymr, int nzmr,
                     const double *sal_planes);
/* <dir>/flowmov/movie_ymean.h5 (axis 1) or movie_zmean.h5 (axis 2): the plane means of
 * mean_yplane / mean_zplane (h5tools/mean_zplane.F90:131-258 / 2-129, averaging by
 * h5tools/means.F90 ymean / zmean / ymeanr / zmeanr), written like the y and z cuts above:
 * planes in afid_gpu_mean_plane's layout (y-mean: nzm x nx; z-mean: nym x nx; vy, vz, temp stored
 * with their nxm rows), sal_planes from afid_gpu_sal_mean_plane (nzmr x nxmr, nymr x nxmr) or
 * NULL.  The reference writes them beside the cuts when nym > 1 and nzm > 1 (main.F90:42,
 * 233-235, 340-343). */
int afid_write_movie_mean(const char *dir, int axis, double tframe, int nframes, const double *times, int nxm,
                          int nym, int nzm, const double *planes, int nxmr, int nymr, int nzmr,
                          const double *sal_planes);

/* ---- spectra ----------------------------------------------------------------------------- */
/* One spectrum file of write_3D_spectrum (h5tools/h5_tools.F90:229-302): dataset 'var' declared
 * with the Fortran dims (nxm, nym, nzm) (C order nzm x nym x nxm); the half spectrum
 * half[nzm][nym/2+1][nxm] (afid_gpu_spectra_read's layout) fills the first nym/2 + 1 wavenumber
 * rows of each z plane and the remaining rows hold 0, the fill value of the reference's
 * hyperslab write. */
int afid_write_spectrum(const char *path, int nxm, int nym, int nzm, const double *half);
/* WriteSpectra (spectra.F90:169-196) through a device context: <dir>/vx_spectrum.h5,
 * vy_spectrum.h5, vz_spectrum.h5, te_spectrum.h5 from the averages of afid_gpu_spectra_update. */
int afid_gpu_write_spectra(afid_ctx_t *ctx, const char *dir);

/* Device context variants (salinity included when afid_gpu_sal_create was called). */
int afid_gpu_write_flow_field(afid_ctx_t *ctx, const char *dir, int final, double save_3d,
                              const afid_continua_master_t *m);
/* Reads, uploads (RK3 history zeroed, salinity re-interpolated) and returns the master's time.
 * When continua_pr.h5 is absent the pressure is uploaded as zero, as the reference leaves it. */
int afid_gpu_read_flow_field(afid_ctx_t *ctx, const char *dir, const afid_continua_master_t *cur,
                             double *time_out);

/* afid_read_flow_interp, then upload (RK3 history zeroed, salinity re-interpolated). */
int afid_gpu_read_flow_interp(afid_ctx_t *ctx, const char *dir, const afid_input_t *in, double *time_out,
                              int *interpolated);

/* afid_run with the restart and save points of the main loop in dir (NULL: same as afid_run).
 * Besides the restart files it writes cordin_info.h5, means.h5 (a sample at start-up and whenever
 * mod(time, TOUT) < dt) and flowmov/movie_{x,y,z}cut.h5 (the cuts at start-up and whenever
 * mod(time, TFRAME) < dt past the first TFRAME), as the reference's main loop does; the samples
 * are written when the run ends, the movie planes kept up to 2 GiB per run.  A restarted run
 * rewrites means.h5 and the movie files with its own samples, where the reference appends to them.
 * NREAD = 1 starts from dir's continua files (time from the master unless IRESET = 1); otherwise
 * from the seeded initial condition.  Frames go to dir/fields, the final continua files to dir
 * on a normal exit (steps done, 333 tmax, 555 ntst). */
int afid_run_io(const afid_input_t *in, int precision, uint64_t seed, int nsteps, int stats_every,
                afid_step_cb cb, void *user, const char *dir, afid_run_stats_t *stats);

#ifdef __cplusplus
}
#endif
#endif /* AFID_CONTINUA_H */
