/*
 * lulesh_b200.h -- C ABI of the B200-native LULESH Lagrange leapfrog step.
 *
 * Plain C types only (no CUDA or torch types): a ctypes / cgo / JNI binding
 * can load liblulesh_b200.so and call these directly.  Every entry point
 * returns a status code (enum lulesh_status) instead of calling exit(), and
 * the reference's exit codes keep their values.
 *
 * Reference interfaces replaced (paths inside varunchotalia/cuda-ipc-benchmarks):
 *   NewDomain                LULESH/cuda/src/lulesh.cu:750-1221
 *   LagrangeLeapFrog         LULESH/cuda/src/lulesh.cu:4438-4452
 *   TimeIncrement            LULESH/cuda/src/lulesh.cu:1400-1461
 *   main loop + checkErrors  LULESH/cuda/src/lulesh.cu:4858-4873, 2879-2892
 *   VerifyAndWriteFinalOutput LULESH/cuda/src/lulesh.cu:4670-4750
 *   write_solution           LULESH/cuda/src/lulesh.cu:4584-4603
 *   Domain field layout      LULESH/cuda/src/lulesh.h:40-298
 *   CommRecv/CommSend/CommSBN/CommSyncPosVel/CommMonoQ
 *                            LULESH/cuda/src/lulesh.h:321-340
 *   error codes              LULESH/cuda/src/lulesh.h:22-26
 *
 * A "set" is everything resident on one GPU that one stream advances:
 *   - one domain (the reference's single-rank run),
 *   - tp^3 subdomains of one problem (the reference's tp^3-rank run, with
 *     the halo exchange done in device memory; "rank" = subdomain index),
 *   - or a batch of independent jobs of different sizes.
 */
#ifndef LULESH_B200_H
#define LULESH_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LULESH_B200_ABI_VERSION 1

/* lulesh.h:22-26 keeps -1/-2/-3; the rest are new, all negative. */
enum lulesh_status {
    LULESH_OK = 0,
    LULESH_VOLUME_ERROR = -1, /* VolumeError: negative element volume   */
    LULESH_QSTOP_ERROR = -2,  /* QStopError: q above qstop              */
    LULESH_FILE_ERROR = -3,   /* LFileError: bad command line / input   */
    LULESH_CUDA_ERROR = -4,   /* a CUDA runtime call failed             */
    LULESH_INVALID_ARG = -5,  /* bad argument (size, index, name, ...)  */
    LULESH_OOM = -6,          /* device memory exhausted / over the cap */
    LULESH_TIMEOUT = -7,      /* a bounded device wait gave up          */
    LULESH_NO_DEVICE = -8,    /* no CUDA device / extension unusable    */
    LULESH_BOUNDS_ERROR = -9  /* -DLULESH_CHECKED builds only: a kernel
                                 index was out of range (replaced by 0) */
};

/* create flags */
#define LULESH_FLAG_MATERIALIZE 0x1 /* also write the per-cycle transients the
                                       reference keeps in Domain (fx/fy/fz,
                                       xdd/ydd/zdd, ql/qq, vnew, delx_*,
                                       delv_*, corner forces) every cycle   */
#define LULESH_FLAG_COMM_STAGED 0x2 /* subdomain sets: exchange halos through
                                       per-message buffers with the
                                       reference's CommSend/CommSBN/
                                       CommSyncPosVel/CommMonoQ sequence
                                       instead of the fused direct kernels */
#define LULESH_FLAG_MIXED 0x4       /* FP32 element-local stress/hourglass/
                                       kinematics arithmetic, compensated
                                       FP32 corner-force sums, FP64 EOS,
                                       node integration and dt              */
#define LULESH_FLAG_HOST_SETUP 0x8  /* build single-domain geometry and
                                       connectivity on the host and copy it
                                       (as NewDomain does) instead of
                                       generating it on the device; the
                                       values are the same either way      */

/* Largest edge of one domain.  Corner forces are indexed
 * elem + padded_numElem * corner in 32-bit integers, as in the reference
 * (Index_t = int32, lulesh.h:32-33, lulesh.cu:2242); at nx = 646 that index
 * passes 2^31 - 1 while the mesh (~157 GB) would still fit in HBM.  Larger
 * jobs are rejected with LULESH_INVALID_ARG; a larger global mesh runs as
 * tp^3 subdomains of at most this edge. */
#define LULESH_MAX_NX 645

/* One sedov job: the reference command line -s -r -b -c -i
 * (LULESH/omp_4.0/lulesh-util.cc:60-173; defaults 30/11/1/1). */
typedef struct lulesh_job {
    int nx;      /* -s: elements per edge of each (sub)domain, 1..645      */
    int numReg;  /* -r: regions (cost model only), >= 1                  */
    int balance; /* -b                                                    */
    int cost;    /* -c                                                    */
    int its;     /* -i: cycle cap; <= 0 runs until time >= stoptime       */
} lulesh_job;

/* Per-job progress, read back from the device. */
typedef struct lulesh_job_state {
    int status;    /* enum lulesh_status of this job                      */
    int bad_elem;  /* element that raised VolumeError/QStopError, or -1   */
    int cycle;     /* cycles completed                                    */
    int done;      /* 1 once time >= stoptime, its reached, or an error   */
    double time;   /* simulated time                                      */
    double deltatime;
    double dtcourant;
    double dthydro;
} lulesh_job_state;

/* Device pointers of one domain, named as the Domain members of
 * lulesh.h:40-298 (node-major nodelist with stride padded_numElem, corner
 * index elem + padded_numElem*corner, delv_* with the ghost-face tail). */
typedef struct lulesh_domain_view {
    int numElem, numNode, padded_numElem, sizeX, sizeY, sizeZ;
    int colLoc, rowLoc, planeLoc, tp, numReg, allElem;
    int numSymmX, numSymmY, numSymmZ;
    int *nodelist, *lxim, *lxip, *letam, *letap, *lzetam, *lzetap, *elemBC;
    int *nodeElemCount, *nodeElemStart, *nodeElemCornerList;
    int *symmX, *symmY, *symmZ, *matElemlist;
    int *regCSR, *regReps, *regNumList, *regElemlist, *regSorted;
    double *e, *p, *q, *ql, *qq, *v, *volo, *delv, *vdov, *arealg, *ss,
        *elemMass;
    double *x, *y, *z, *xd, *yd, *zd, *xdd, *ydd, *zdd, *fx, *fy, *fz,
        *nodalMass;
    double *vnew, *delx_xi, *delx_eta, *delx_zeta, *delv_xi, *delv_eta,
        *delv_zeta, *fx_elem, *fy_elem, *fz_elem;
} lulesh_domain_view;

typedef struct lulesh_set lulesh_set;

/* ---- lifetime -------------------------------------------------------- */

/* Replaces NewDomain (lulesh.cu:750) for one problem decomposed into tp^3
 * subdomains of job->nx^3 elements each (tp = 1: the single-domain run).
 * Subdomain r sits at col = r % tp, row = (r / tp) % tp, plane = r / tp^2
 * (InitMeshDecomp, lulesh.cu:4606-4668) and seeds its regions with
 * srand(r) (lulesh.cu:1263-1270).  All device memory comes from one arena
 * owned by the set.  `device` < 0 keeps the current device. */
int lulesh_create(const lulesh_job *job, int tp, int flags, int device,
                  lulesh_set **out);

/* A batch of independent single-domain jobs advanced together; each keeps
 * its own dt, time, cycle cap and status.  No reference counterpart: the
 * reference runs one job per process. */
int lulesh_create_batch(const lulesh_job *jobs, int njobs, int flags,
                        int device, lulesh_set **out);

/* Replaces NewDomain's unstructured branch (lulesh.cu:855-1052, the `-u
 * file.lmesh` run): one FP64 domain read from an lmesh file ("E N" header,
 * N coordinate lines, E lines of 8 node ids, E lines of 6 face links, then
 * the symmX/Y/Z and free-surface node sets, each a count followed by ids).
 * job->nx is ignored; numReg/balance/cost/its keep their meaning.  The
 * energy deposit goes to the element whose three minus faces carry
 * symmetry, and free-surface faces carry the *_FREE boundary bits.
 * Returns LULESH_FILE_ERROR for an unreadable or malformed file, and
 * LULESH_INVALID_ARG with LULESH_FLAG_COMM_STAGED or LULESH_FLAG_MIXED. */
int lulesh_create_from_mesh(const char *path, const lulesh_job *job,
                            int flags, int device, lulesh_set **out);

/* Frees the arena, graphs and streams (the reference's teardown,
 * lulesh.cu:4904-4944, minus MPI). */
int lulesh_destroy(lulesh_set *set);

/* Bytes of device memory a set of these jobs would hold (the admission
 * model of the serving loop). */
size_t lulesh_footprint_bytes(const lulesh_job *jobs, int njobs, int tp);

/* ---- stepping -------------------------------------------------------- */

/* Use this stream (a cudaStream_t passed as void*) for all later work;
 * NULL makes the set create and own one. */
int lulesh_set_stream(lulesh_set *set, void *stream);

/* One cycle of TimeIncrement + LagrangeLeapFrog for every job in the set,
 * enqueued asynchronously as a captured CUDA graph (lulesh.cu:4438-4452
 * with TimeIncrement moved onto the device).  Jobs that are done skip. */
int lulesh_lagrange_leapfrog(lulesh_set *set);

/* `ncycles` such cycles, asynchronously.  On a stream the caller is
 * capturing into its own CUDA graph, the cycles' kernels are enqueued one
 * by one and become nodes of that graph; make one lulesh_step(set, 0) call
 * before the capture (it prepares the set outside the capture), or the
 * call returns LULESH_INVALID_ARG.  ncycles = 0 only prepares. */
int lulesh_step(lulesh_set *set, int ncycles);

/* The whole run in one CUDA graph launch: a WHILE conditional node repeats
 * the cycle until every job of the set is done (the reference's host loop,
 * lulesh.cu:4858-4873, moved onto the device).  max_cycles bounds the loop
 * (<= 0: 1,000,000 cycles); jobs still running when it stops are left as
 * they are.  Synchronous; returns like lulesh_run. */
int lulesh_run_graph(lulesh_set *set, long long max_cycles);

/* Capture k consecutive cycles in one CUDA graph (default 1): lulesh_step(n)
 * then issues n / k launches of the k-cycle graph and n % k of the
 * one-cycle graph, so a whole batch run can be a single graph launch. */
int lulesh_set_graph_cycles(lulesh_set *set, int k);

/* Checkpoint of a set's whole state: every device array of every domain
 * and the time state of every job, behind a header that identifies the
 * set's jobs, subdomain count and flags.  No reference counterpart (the
 * reference has no restart path).  A checkpoint loads only into a set
 * created with the same jobs, tp and flags (else LULESH_INVALID_ARG);
 * stepping on from a loaded checkpoint gives the same results, bit for
 * bit, as stepping on from where it was saved.  Both calls synchronise the
 * set's stream. */
size_t lulesh_checkpoint_bytes(const lulesh_set *set);
int lulesh_checkpoint_save(lulesh_set *set, void *host_buf, size_t bytes);
int lulesh_checkpoint_load(lulesh_set *set, const void *host_buf, size_t bytes);

/* Launch shapes of a set.  No reference counterpart (the reference launches
 * fixed 64/128-thread blocks per kernel); results do not depend on them. */
typedef struct lulesh_tuning {
    int elem_block;   /* elements (threads) per block of the FP64 force,
                         kinematics and EOS kernels: 64, 128 or 256 */
    int node_block;   /* nodes (threads) per block of the nodal kernel:
                         128, 256 or 512 */
    int order;        /* block tables: 0 domains in creation order,
                         1 largest domain first */
    int graph_cycles; /* cycles per graph launch, >= 1 */
} lulesh_tuning;

typedef struct lulesh_tune_trial {
    lulesh_tuning tuning;
    double ms_per_cycle; /* best of the rounds, device time */
} lulesh_tune_trial;

int lulesh_get_tuning(const lulesh_set *set, lulesh_tuning *out);

/* Apply launch shapes.  Sets of subdomains (tp > 1), staged-comm and mixed
 * precision sets take only elem_block = node_block = 128.
 * LULESH_INVALID_ARG for a shape outside the lists above. */
int lulesh_set_tuning(lulesh_set *set, const lulesh_tuning *tuning);

/* Autotuner (no reference counterpart): saves the set's device state,
 * times every candidate shape for `trial_cycles` cycles from that same state
 * (`rounds` times each, interleaved; best kept), first over elem_block x
 * node_block x order at one cycle per launch, then graph_cycles in
 * {1, 2, 4, 8, 16} for the winner; restores the state and applies the
 * fastest.  Synchronous; needs device memory for one copy of the set's
 * state.  The trials (up to max_trials) are written to `trials`. */
int lulesh_autotune(lulesh_set *set, int trial_cycles, int rounds, lulesh_tuning *best,
                    lulesh_tune_trial *trials, int max_trials, int *n_trials);

/* The reference main loop (lulesh.cu:4858-4873): cycles until every job
 * has reached its cap or stoptime or failed, checking status every
 * `check_every` cycles (<= 0: 64).  Synchronous.  Returns LULESH_OK or the
 * first job error (VolumeError / QStopError as the reference's exit code). */
int lulesh_run(lulesh_set *set, int check_every);

/* One cycle driven from the host the way the reference drives it: the
 * host passes the time state in (host buffer, copied H2D), the device runs
 * one cycle, and the new time state plus status come back (D2H) into
 * `out`.  in may be NULL to continue from the device state.  Used for the
 * end-to-end measurement; synchronous. */
int lulesh_host_cycle(lulesh_set *set, const lulesh_job_state *in,
                      lulesh_job_state *out);

/* Block until queued work is done; returns the first CUDA error seen. */
int lulesh_sync(lulesh_set *set);

/* Profiling: run `ncycles` cycles launching each phase on its own with CUDA
 * events around it (on the set's stream), and return the average duration
 * in milliseconds of each phase in ms_out[0..*nphases-1], named by
 * lulesh_phase_name().  No reference counterpart (the reference times the
 * whole loop, lulesh.cu:4851-4886). */
int lulesh_profile_phases(lulesh_set *set, int ncycles, double *ms_out, int *nphases);
const char *lulesh_phase_name(int phase);
#define LULESH_MAX_PHASES 12

/* ---- results --------------------------------------------------------- */

int lulesh_num_jobs(const lulesh_set *set);
int lulesh_num_domains(const lulesh_set *set);
int lulesh_job_state_get(lulesh_set *set, int job, lulesh_job_state *out);

/* e[octantCorner] of the job's origin domain (lulesh.cu:4700-4710). */
int lulesh_origin_energy(lulesh_set *set, int job, double *energy);

/* Plane-0 symmetry check of the job's origin domain (lulesh.cu:4712-4736). */
int lulesh_symmetry(lulesh_set *set, int job, double *max_abs,
                    double *total_abs, double *max_rel);

/* Copy a named Domain field of one domain to/from host memory.  `nbytes`
 * must equal the field's size (lulesh_field_bytes). */
int lulesh_field_bytes(lulesh_set *set, int domain, const char *name,
                       size_t *nbytes);
int lulesh_get_field(lulesh_set *set, int domain, const char *name,
                     void *host_dst, size_t nbytes);
int lulesh_set_field(lulesh_set *set, int domain, const char *name,
                     const void *host_src, size_t nbytes);

/* Device pointers of one domain (valid until lulesh_destroy). */
int lulesh_domain_view_get(lulesh_set *set, int domain,
                           lulesh_domain_view *out);

/* Write xyz.asc-format node coordinates of one domain (lulesh.cu:4584). */
int lulesh_write_solution(lulesh_set *set, int domain, const char *path);

const char *lulesh_status_string(int status);
const char *lulesh_last_error(void);

/* FP64 throughput of a GPU (device < 0: the current one), measured: fused
 * multiply-adds per second (one FMA counts once) of independent
 * register-only FMA chains over every SM, best of three timed launches.
 * The denominator of the FP64 rooflines the benchmark reports.  No
 * reference counterpart. */
int lulesh_measure_fp64_peak(int device, double *fma_per_s);

/* ---- serving: continuous batching of sedov jobs ----------------------- */
/* No reference counterpart (the reference runs one job per process).  A
 * server owns one GPU stream.  Submitted jobs are meshed on host worker
 * threads, admitted in arrival order while their device footprint
 * (lulesh_footprint_bytes) fits under hbm_cap_bytes and a slot is free,
 * and from then on keep their Domain state resident on the device.  Each
 * lulesh_server_step advances every resident job by cycles_per_step cycles
 * in one captured graph (jobs of different sizes share every launch),
 * retires the jobs that finished (time >= stoptime, its reached, or an
 * error) and admits new ones.  A job's result is bit-identical to running
 * it alone with lulesh_create + lulesh_run. */
typedef struct lulesh_server_config {
    size_t hbm_cap_bytes; /* admission cap on the device memory of resident jobs */
    int max_jobs;         /* resident jobs at most (slots), >= 1 */
    int cycles_per_step;  /* cycles per lulesh_server_step, >= 1 */
    int prepare_threads;  /* host threads that build submitted meshes, >= 1 */
    int device;           /* < 0: current device */
} lulesh_server_config;

typedef struct lulesh_server_result {
    long long id;          /* as returned by lulesh_server_submit */
    int status;            /* LULESH_OK or VolumeError / QStopError */
    int cycle;             /* cycles run */
    int bad_elem;          /* element of the error, or -1 */
    double origin_energy;  /* Final Origin Energy */
    double time;           /* simulated time reached */
    double t_submit, t_admit, t_done; /* host monotonic clock, seconds */
} lulesh_server_result;

typedef struct lulesh_server lulesh_server;

int lulesh_server_create(const lulesh_server_config *cfg, lulesh_server **out);
int lulesh_server_destroy(lulesh_server *srv);
/* Queue a job (returns immediately; meshing starts on a worker thread). */
int lulesh_server_submit(lulesh_server *srv, const lulesh_job *job, long long *id);
/* Retire finished jobs, admit queued ones that fit, advance the resident
 * ones.  *n_active / *n_queued (may be NULL) report the state after it. */
int lulesh_server_step(lulesh_server *srv, int *n_active, int *n_queued);
/* Move up to `max` finished results into out[]; *n receives the count. */
int lulesh_server_poll(lulesh_server *srv, lulesh_server_result *out, int max, int *n);
/* Host monotonic clock used for the t_* fields (seconds). */
double lulesh_server_clock(void);

/* ---- nodal forces without allocation --------------------------------- */
/* No counterpart in the reference.  For callers that cannot allocate device
 * memory -- a host code whose memory manager owns the whole GPU budget, or a
 * latency-sensitive loop that cannot afford cudaMalloc/cudaFree, which
 * synchronise the device -- this computes the nodal forces fx/fy/fz of one
 * structured domain of nx^3 elements (stress + FB hourglass corner forces
 * summed per node in corner order, as CalcVolumeForceForElems does) from
 * caller-owned device arrays in the Domain layout: x..zd over (nx+1)^3
 * nodes, volo/v/p/q/ss/elemMass over nx^3 elements.  hgcoef is the
 * hourglass coefficient (3.0 in the reference).  *bad_elem (device int,
 * may be NULL) receives the smallest element with a negative volume, or -1.
 *
 * It allocates nothing: its only scratch is one fixed device array of
 * LULESH_NOALLOC_MAX_ELEMS elements' corner forces (6 MiB) that every GPU
 * which loads the library holds until the process exits.  nx above
 * LULESH_NOALLOC_MAX_NX is rejected with LULESH_INVALID_ARG and a message in
 * lulesh_last_error().  The first call on a device looks up that array's
 * device address (with the device current), so make the first call on each
 * device before any stream capture.  A device reset (cudaDeviceReset) or a
 * context the caller created itself moves the array, so every call made
 * outside stream capture looks the address up again; a call on a capturing
 * stream reuses the address of the last call outside capture, so after a
 * reset make one call outside capture first.  All calls share the one array and it
 * keeps the last call's contents: calls that overlap on the GPU (different
 * streams, or different host threads, on the same device) race with each
 * other; serialise them on one stream.  Asynchronous on `stream`
 * (a cudaStream_t, NULL for the legacy default stream). */
#define LULESH_NOALLOC_MAX_NX 32
#define LULESH_NOALLOC_MAX_ELEMS (LULESH_NOALLOC_MAX_NX * LULESH_NOALLOC_MAX_NX * LULESH_NOALLOC_MAX_NX)
int lulesh_volume_force_noalloc(int nx, const double *x, const double *y, const double *z,
                                const double *xd, const double *yd, const double *zd,
                                const double *volo, const double *v, const double *p,
                                const double *q, const double *ss, const double *elemMass,
                                double hgcoef, double *fx, double *fy, double *fz,
                                int *bad_elem, void *stream);

/* ---- comm backend (lulesh.h:321-340; comm/comm_backend.h:7-22) ------- */
/* msgType: 1024 MSG_COMM_SBN, 2048 MSG_SYNC_POS_VEL, 3072 MSG_MONOQ
 * (lulesh.h:314-317).  Fields are named by Domain member id below.  `rank`
 * is a subdomain index of the set, or -1 for every subdomain in one launch.
 * These run on the set's stream and order like the reference: all ranks'
 * CommRecv, then CommSend, then the unpack (CommSBN / CommSyncPosVel /
 * CommMonoQ).  A single-domain set returns LULESH_OK without work, as the
 * reference does when numRanks() == 1 (lulesh-comms.cu:65-66). */
enum lulesh_field_id {
    LULESH_F_X = 0, LULESH_F_Y, LULESH_F_Z, LULESH_F_XD, LULESH_F_YD,
    LULESH_F_ZD, LULESH_F_FX, LULESH_F_FY, LULESH_F_FZ, LULESH_F_NODALMASS,
    LULESH_F_DELV_XI, LULESH_F_DELV_ETA, LULESH_F_DELV_ZETA,
    /* moved only by the exchange between GPUs below (not Comm* fields) */
    LULESH_F_FX_ELEM, LULESH_F_FY_ELEM, LULESH_F_FZ_ELEM, LULESH_F_VOLO
};
#define LULESH_MSG_COMM_SBN 1024
#define LULESH_MSG_SYNC_POS_VEL 2048
#define LULESH_MSG_MONOQ 3072
#define LULESH_MAX_FIELDS_PER_COMM 6

int lulesh_comm_recv(lulesh_set *set, int rank, int msgType, int xferFields,
                     int dx, int dy, int dz, int doRecv, int planeOnly);
int lulesh_comm_send(lulesh_set *set, int rank, int msgType, int xferFields,
                     const int *fieldIds, int dx, int dy, int dz, int doSend,
                     int planeOnly);
int lulesh_comm_sbn(lulesh_set *set, int rank, int xferFields,
                    const int *fieldIds);
int lulesh_comm_sync_posvel(lulesh_set *set, int rank);
int lulesh_comm_monoq(lulesh_set *set, int rank);

/* Offset (in doubles) inside rank recvRank's receive buffer where the
 * message from direction (dCol,dRow,dPlane) lands: the posting-order
 * contract of comm_backend.h:75-138.  Returns -1 if no such message. */
long lulesh_comm_recv_offset(lulesh_set *set, int recvRank, int dCol,
                             int dRow, int dPlane, int xferFields, int doRecv,
                             int planeOnly);

/* ---- one problem over several GPUs ------------------------------------ */
/* The reference's multi-rank run (one rank per GPU, halos over MPI / CUDA
 * IPC / NVSHMEM: LULESH/cuda/README.md:18-113, lulesh-comms-direct.cu:
 * 50-404, comm/comm_ipc_common.h:26-261) as parts: the tp^3 subdomains of
 * one problem are split over `nparts` GPUs, one process (and one set) per
 * GPU; rank r belongs to part lulesh_part_of(r, tp, nparts) = r * nparts /
 * tp^3.  A subdomain whose neighbour sits on another part reads that
 * neighbour through a proxy: arrays in the neighbour's layout whose boundary
 * layers the messages below fill.  The cycle's kernels are those of an
 * in-device subdomain set, so a decomposed run gives the single-domain
 * results bit for bit, like the in-device 2x2x2 run.
 *
 * Messages (kind, from part, to part) are planned by lulesh_halo_plan: item
 * i is field[i] of subdomain rank[i] at index[i], and lands at the same
 * index of the receiver's proxy of that subdomain.  Kinds:
 *   CORNERS  corner forces of the element layers facing the receiver
 *            (replaces CommSend/CommSBN of fx/fy/fz, lulesh.cu:2897-2921:
 *            the receiver adds every node's corners in corner order, so no
 *            partial sums and no float atomics cross)
 *   POSVEL   x..zd of the node layers facing a receiver on the minus sides
 *            (CommSyncPosVel, lulesh.cu:3061-3094)
 *   MONOQ    delv_xi/eta/zeta of the element face layers (CommMonoQ,
 *            lulesh.cu:4165-4190)
 *   MASS     volo of the element layers, once at set-up (the init-time
 *            nodalMass CommSBN, lulesh.cu:4811-4831)
 * The host functions (lulesh_part_of, lulesh_halo_peers, lulesh_halo_plan)
 * need no GPU. */
#define LULESH_HALO_CORNERS 0
#define LULESH_HALO_POSVEL 1
#define LULESH_HALO_MONOQ 2
#define LULESH_HALO_MASS 3

int lulesh_part_of(int rank, int tp, int nparts);
/* The parts that `part` exchanges messages with, ascending, into peers[]
 * (up to max_peers); returns their number or a negative status. */
int lulesh_halo_peers(int tp, int nparts, int part, int *peers, int max_peers);
/* Plan of one message; returns the number of items (the message length in
 * doubles) and fills up to max_items of rank/field/index (each may be
 * NULL), or a negative status. */
long long lulesh_halo_plan(int nx, int tp, int nparts, int from_part, int to_part, int kind,
                           int *rank, int *field, long long *index, long long max_items);

/* This GPU's part of the problem: the subdomains it owns (domains
 * 0..n-1 of the set in rank order) and proxies of their neighbours on other
 * parts.  Before the first cycle, exchange the MASS messages with every
 * peer (pack, move, unpack) and call lulesh_part_finish_setup, which sums
 * each node's mass over the elements of the whole problem that touch it,
 * on the device.  nparts = 1 gives an ordinary subdomain set.  FP64 and
 * the fused exchange only (no LULESH_FLAG_MIXED / LULESH_FLAG_COMM_STAGED);
 * a part of several GPUs advances through lulesh_part_phase, not
 * lulesh_step. */
int lulesh_create_part(const lulesh_job *job, int tp, int nparts, int part, int flags,
                       int device, lulesh_set **out);
int lulesh_part_finish_setup(lulesh_set *set);

/* Length in doubles of the message of `kind` this part sends to
 * (to_peer = 1) or receives from (to_peer = 0) part `peer`. */
long long lulesh_halo_count(lulesh_set *set, int kind, int peer, int to_peer);
/* Enqueue on the set's stream: gather the message for `peer` into dev_buf,
 * or scatter the message received from `peer` into the proxies.  dev_buf
 * is caller-owned device memory of lulesh_halo_count doubles. */
int lulesh_halo_pack(lulesh_set *set, int kind, int peer, double *dev_buf);
int lulesh_halo_unpack(lulesh_set *set, int kind, int peer, const double *dev_buf);

/* One phase of the cycle, enqueued on the set's stream.  A cycle of a part
 * is: TIME_INCREMENT, FORCE, exchange CORNERS, NODAL, [exchange POSVEL,
 * POSVEL_SYNC,] KINEMATICS, exchange MONOQ, MONOQ_GHOST, EOS, then the dt
 * reduction below.  The POSVEL exchange and its sync may be left out (the
 * part computes its shared nodes exactly as their owner does).
 * MONOQ_GHOST enqueues nothing in this build: the EOS reads the
 * neighbours' delv layers in the proxies the MONOQ messages filled. */
#define LULESH_PHASE_TIME_INCREMENT 0
#define LULESH_PHASE_FORCE 1
#define LULESH_PHASE_NODAL 2
#define LULESH_PHASE_POSVEL_SYNC 3
#define LULESH_PHASE_KINEMATICS 4
#define LULESH_PHASE_MONOQ_GHOST 5
#define LULESH_PHASE_EOS 6
int lulesh_part_phase(lulesh_set *set, int phase);

/* The dt reduction of TimeIncrement (MPI_Allreduce MIN, lulesh.cu:
 * 1423-1429) and the error flags of checkErrors: dt_pack writes this
 * part's four int64 values (courant and hydro dt minima as IEEE bit
 * patterns, the smallest element with a volume error and with q above
 * qstop, INT_MAX for none) to dev_buf; the caller takes the element-wise
 * minimum over all parts (e.g. ncclAllReduce MIN on int64) and hands the
 * result to dt_unpack before the next TIME_INCREMENT. */
int lulesh_part_dt_pack(lulesh_set *set, long long *dev_buf);
int lulesh_part_dt_unpack(lulesh_set *set, const long long *dev_buf);

/* Direct transport (peer stores over NVLink): every part owns a mailbox
 * that holds each message it receives plus one arrival flag per message;
 * the sender's kernel stores its message straight into the receiver's
 * mailbox and then raises the flag to a sequence number, and the receiver's
 * kernel waits for that number (bounded) before scattering the message into
 * its proxies.  This is the reference's remote-pack IPC backend with its
 * token protocol (comm/comm_ipc_common.h:26-261, lulesh-comms-direct.cu:
 * 241-404) with the tokens in device memory.  The mailbox layout follows
 * from the plan, so a sender knows where its message lands.
 *   lulesh_part_mailbox: this part's mailbox (device pointer, size) and,
 *     if ipc_handle is not NULL, its cudaIpcMemHandle (64 bytes) for the
 *     peers' processes;
 *   lulesh_part_set_peer_mailbox: a peer's mailbox, as a device pointer
 *     (parts in one process) or an IPC handle (opened with peer access);
 *   lulesh_halo_put: enqueue the message of `kind` to `peer` and raise its
 *     flag to `seq` (every exchange of a kind uses the next number, from 1);
 *   lulesh_halo_take: enqueue the wait for `seq` from `peer` (at most
 *     timeout_ms; on timeout the job stops with LULESH_TIMEOUT and nothing
 *     is scattered) and the scatter.
 * A mailbox is reused every cycle: a sender may put the next message of a
 * kind only after the receiver has taken the previous one, which the
 * per-cycle dt reduction (a collective over all parts) guarantees. */
int lulesh_part_mailbox(lulesh_set *set, void **dev_ptr, size_t *bytes, void *ipc_handle);
int lulesh_part_set_peer_mailbox(lulesh_set *set, int peer, const void *dev_ptr,
                                 const void *ipc_handle);
int lulesh_halo_put(lulesh_set *set, int kind, int peer, unsigned int seq);
int lulesh_halo_take(lulesh_set *set, int kind, int peer, unsigned int seq, double timeout_ms);

/* Bounded wait on a device flag for transports that signal arrival with a
 * flag the sender sets in this GPU's memory (peer stores): enqueues a
 * one-thread kernel that spins until *flag >= expect or timeout_ms has
 * passed; on timeout the set's job is stopped with status LULESH_TIMEOUT
 * (read by lulesh_job_state_get) and the kernel returns, so the context
 * stays usable. */
int lulesh_wait_flag(lulesh_set *set, const unsigned int *dev_flag, unsigned int expect,
                     double timeout_ms);

#ifdef __cplusplus
}
#endif
#endif /* LULESH_B200_H */
