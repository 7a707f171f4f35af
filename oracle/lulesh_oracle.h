/*
 * lulesh_oracle.h -- CPU oracle for the LULESH Lagrange leapfrog step.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py as the checker.  The product never links it.
 *
 * The oracle restates, in plain C with no FMA contraction, the arithmetic of
 * the reference CUDA single-domain build (LULESH/cuda/src/lulesh.cu).  Parity
 * pins: the reference omp_4.0 CPU build and the reference CUDA build, both
 * compiled from the unmodified reference sources into oracle/_ref/, plus the
 * reference's published Final Origin Energies (results/lulesh_results.csv,
 * ucx_lulesh_experiments_46508.csv).
 */
#ifndef LULESH_ORACLE_H
#define LULESH_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleDomain OracleDomain;

/* Build one structured domain exactly as NewDomain (lulesh.cu:750-1221):
 * nx elements per edge, tp^3 decomposition with this domain at
 * (col,row,plane) and region seed `rank` (srand(rank), lulesh.cu:1263-1270).
 * A single domain is tp=1, col=row=plane=rank=0. */
OracleDomain *oracle_create(int nx, int numReg, int balance, int cost,
                            int tp, int col, int row, int plane, int rank);
/* One unstructured domain read from an lmesh file, as the -u branch of
 * NewDomain reads it (lulesh.cu:855-1052), with the two corrections the
 * product makes: free-surface faces carry the *_FREE bits, and the energy
 * 3.948746e7 stays at the octant corner (the initial dt follows from that
 * element's volume).  NULL for an unreadable or malformed file. */
OracleDomain *oracle_create_lmesh(const char *path, int numReg, int balance,
                                  int cost);
void oracle_destroy(OracleDomain *d);

/* One cycle: TimeIncrement then LagrangeLeapFrog (lulesh.cu:4438-4452,
 * with TimeIncrement hoisted as lulesh.cu:2905 does).  Returns 0, or -1
 * (VolumeError) / -2 (QStopError) after the cycle that raised it. */
int oracle_step(OracleDomain *d);

/* The main loop of lulesh.cu:4858-4873: until time >= stoptime or `its`
 * cycles (its < 0: no cap).  Returns the status of the last cycle; the
 * number of cycles run is stored in *cycles_run. */
int oracle_run(OracleDomain *d, int its, int *cycles_run);

/* Field access: pointer to the named array and its element count
 * (doubles for real fields, ints for index fields).  Names follow the
 * Domain members of lulesh.h:40-298. */
double *oracle_real_field(OracleDomain *d, const char *name, int *count);
int *oracle_int_field(OracleDomain *d, const char *name, int *count);

/* Scalars: "time", "deltatime", "dtcourant", "dthydro", "cycle",
 * "numElem", "numNode", "padded_numElem", "numReg", "bad_vol", "bad_q",
 * "numSymmX", "numSymmY", "numSymmZ", "initial_deltatime". */
double oracle_scalar(OracleDomain *d, const char *name);
void oracle_set_deltatime(OracleDomain *d, double dt);

/* ---- decomposed stepping -------------------------------------------- */
/* One subdomain of a tp^3 problem stepped phase by phase, reading its
 * neighbours through mirrors: arrays in each neighbour's own layout (the
 * neighbour's real arrays, or copies of whatever parts a halo exchange has
 * filled).  Used to check an exchange between processes on the CPU: with
 * every mirror holding what the neighbour holds, a decomposed run gives the
 * single-domain values bit for bit (node sums in corner order over the
 * whole mesh, nodal mass in ascending global element order). */
typedef struct OracleMirror {
    const double *x, *y, *z, *xd, *yd, *zd;
    const double *fx_elem, *fy_elem, *fz_elem;
    const double *delv_xi, *delv_eta, *delv_zeta;
    const double *volo;
} OracleMirror;

#define ORACLE_PHASE_TIME_INCREMENT 0
#define ORACLE_PHASE_FORCE 1       /* corner forces only */
#define ORACLE_PHASE_NODAL 2       /* node sums (mirrors) + node update */
#define ORACLE_PHASE_POSVEL_SYNC 3 /* x..zd from the +side owner */
#define ORACLE_PHASE_KINEMATICS 4
#define ORACLE_PHASE_MONOQ_GHOST 5 /* delv_* ghost faces from mirrors */
#define ORACLE_PHASE_EOS 6         /* monoQ region, EOS, dt constraints */

/* dir = (dx+1) + 3(dy+1) + 9(dz+1); m NULL clears (the copy of the struct
 * is kept; the arrays must outlive the stepping) */
void oracle_set_mirror(OracleDomain *d, int dir, const OracleMirror *m);
int oracle_phase(OracleDomain *d, int phase);
void oracle_nodal_mass_decomposed(OracleDomain *d);
/* the dt minima the next TIME_INCREMENT uses (after a reduction over
 * subdomains) */
void oracle_set_dt_minima(OracleDomain *d, double dtcourant, double dthydro);

/* VerifyAndWriteFinalOutput numbers (lulesh.cu:4700-4736). */
double oracle_origin_energy(OracleDomain *d);
void oracle_symmetry(OracleDomain *d, double *max_abs, double *total_abs,
                     double *max_rel);

#ifdef __cplusplus
}
#endif
#endif
