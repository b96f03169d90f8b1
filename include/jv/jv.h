/*
 * jv.h -- C ABI of libjv, a single-GPU (NVIDIA B200, sm_100a) elastic 3D
 * staggered-grid FDTD modelling and VOWR reverse-time-migration library.
 *
 * It is a drop-in for the modelling and RTM calls of the jarvis
 * `fdtd3d_blend_elastic_model_mpi` modules.  The reference exposes those
 * calls as C++ template classes driven by one cross-compiler function;
 * each entry point below names the reference interface it replaces
 * (paths relative to the reference project root;
 *  FD  = src/jarvis_cpp/jarvis/.jarvis_2_app/.jarvis_3_seismology/elastic_1_fdtd3d_model_mpi,
 *  RTM = src/jarvis_cpp/jarvis/.jarvis_2_app/.jarvis_3_seismology/elastic_1_rtm3d_model_mpi).
 *
 * Conventions
 *  - Grids are the reference's Frame: x fastest ("rows"), then y ("cols"),
 *    then z ("slices").  Model arrays and images cover gridphy
 *    (nx*ny*nz floats); the library adds `pml` cells per face (gridext).
 *  - Positions are metres in the reference's convention (gridphy origin at
 *    0, node k at k*d); points outside gridphy are dropped as the
 *    reference's SubGeometry does.
 *  - Traces are [n_recv][nt] float32, time fastest.
 *  - Every call returns a jv_status; no call aborts the process.  The
 *    message of the last failure on the calling thread is available from
 *    jv_last_error().
 *  - A context is bound to one CUDA device and one stream; calls on one
 *    context must not overlap (distinct contexts are independent).
 *  - `*_device` entry points take device pointers (no host copies); the
 *    others take host pointers and do the copies inside the call.
 */
#ifndef JV_JV_H
#define JV_JV_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define JV_ABI_VERSION 1

typedef enum jv_status {
    JV_OK = 0,
    JV_EINVAL = -1,    /* bad argument / unsupported problem                */
    JV_ENOMEM = -2,    /* device or host allocation failed                  */
    JV_ECUDA = -3,     /* a CUDA runtime call failed                        */
    JV_EIO = -4,       /* file missing / unreadable / malformed             */
    JV_ETIMEOUT = -5,  /* a bounded wait ran out                            */
    JV_ECANCELED = -6, /* job cancelled                                     */
    JV_ESTATE = -7,    /* call not valid in the context's current state     */
    JV_ENOTSUP = -8    /* feature not built / not supported on this device  */
} jv_status;

typedef struct jv_ctx jv_ctx;

/* gridphy and spacing: the fields of Frame gridphy plus pml_num
 * (.jarvis_0_meta/.jarvis_2_field/jarvis_0_frame_bones.hpp:9-51;
 *  FD/fdtd3d_0_base_module/fdtd3d_base_1_interface.hpp:41). */
typedef struct jv_grid {
    int nx, ny, nz; /* gridphy cells; each >= 8                          */
    int pml;        /* cells added per face; 4 <= pml                    */
    float dx, dy, dz;
} jv_grid;

/* Storage precision of the VOWR boundary store: JV_BF16 / JV_FP16 keep each
 * stored value as value/scale in 16 bits, with one FP32 scale per face box
 * and time step (the box's largest magnitude). Wavefields stay FP32, and all
 * arithmetic is FP32. */
typedef enum jv_precision { JV_FP32 = 0, JV_BF16 = 1, JV_FP16 = 2 } jv_precision;

/* Boundary-store placement for VOWR: DEVICE = HBM (JV_ENOMEM beyond
 * store_budget), HOST = pinned host memory mapped into the device (the pack
 * and unpack kernels cross the host link), AUTO = the device when the store
 * fits, else the host. */
typedef enum jv_store_mode { JV_STORE_AUTO = 0, JV_STORE_DEVICE = 1, JV_STORE_HOST = 2 } jv_store_mode;

typedef struct jv_options {
    int device;         /* CUDA device ordinal                                   */
    int rec_width;      /* GeoConst::rec_width, 1..4 (0 -> 1)                    */
    int precision;      /* jv_precision                                          */
    int store_mode;     /* jv_store_mode                                         */
    int use_graphs;     /* capture the time loop in CUDA graphs (default on)     */
    int graph_steps;    /* time steps per captured graph (0 -> library default)  */
    size_t store_budget;/* max bytes of HBM for the boundary store (0 -> auto)   */
    int kernel_variant; /* stencil kernels: 0 one plane per block, 1 z-marching, 2 x-vectorised,
                           3 as 2 with a TMA-fed z-marching stress update, 4 (default) as 3
                           with the absorbing layers' stress update in the same TMA kernel
                           (even pml_num and nx; other grids run variant 3's kernels);
                           -1: measured choice among 4, 3, 2, variant 4's run chunking,
                           the absorbing-layer register budget and the float4 kernels'
                           block shape on this grid at creation, kept per grid shape;
                           jv_get_kernel_config reports it */
    int zchunk;         /* z planes per block for variant 1 (0 -> auto)          */
    int tile_gx;        /* variant 2: 4-cell x groups per block (0 -> auto)      */
    int tile_gy;        /* variant 2: rows per block (0 -> auto)                 */
    int min_blocks;     /* interior kernels: register budget for 3 or 4 blocks/SM (0 -> 4) */
    int pml_min_blocks; /* absorbing-layer kernels: the same (0 -> 4)            */
    int planes_per_thread;     /* variant 2: z planes a thread updates, 1 or 2 (0 -> 1) */
    int pml_planes_per_thread; /* absorbing-layer kernels: the same (0 -> 1)      */
    int run_chunks;     /* variant 4: chunks each tile's planes are cut into for the
                           persistent kernels' run schedule (0 -> the cost model's
                           choice; with kernel_variant -1 the measured choice among the
                           cost model's three best); jv_get_kernel_config reports it */
    int autotune;       /* 1 (default): at creation, time the knobs that cannot change a result --
                           variant 4's run chunking among the cost model's three best and the
                           float4 kernels' block shape -- on this grid and keep the fastest, per
                           grid shape and device for the process (skipped when run_chunks,
                           tile_gx or tile_gy fix them, or kernel_variant is -1, which makes the
                           wider choice); 0: the cost model's chunking and the default shape */
} jv_options;

/* Fills `o` with the defaults (device 0, rec_width 1, FP32, auto store,
 * graphs on). */
void jv_options_default(jv_options *o);


/* Creates a context from host model arrays on gridphy (vp, vs, rho).
 * Replaces elasticGeoModel<global/local>::initialize
 * (FD/fdtd3d_0_base_module/fdtd3d_base_3_geomodel_meat.hpp:405-577) with the
 * model given in memory; dt, fm and nt are ArgList::dt, fm and
 * ceil(T/dt) (FD/fdtd3d_0_base_module/fdtd3d_base_4_seisrecord_meat.hpp:
 * 273-285). */
jv_status jv_create(const jv_grid *grid, const float *vp, const float *vs, const float *rho, float dt, float fm,
                    int nt, const jv_options *opt, jv_ctx **out);

/* Reads a reference project directory: proj_path + "argfile.json" (the
 * ArgList schema, FD/fdtd3d_0_base_module/fdtd3d_base_1_interface.hpp:50-112),
 * shot/rece geometry (src/jarvis_cpp/jarvis/.jarvis_1_util/.jarvis_2_geometry/
 * jarvis_device_geometry_meat.hpp:6-128) and model_path (.gms with vp, vs,
 * rho, src/jarvis_cpp/jarvis/.jarvis_1_util/.jarvis_0_gms/
 * jarvis_device_gms_meat.hpp:11-79).  x/y/z_divide_num must be 1.  The
 * optional argfile keys "rec_width" and "precision" override opt. */
jv_status jv_open(const char *proj_path, const jv_options *opt, jv_ctx **out);

/* The argfile of a reference project directory as ArgList::mpi_read_arg_file
 * reads it (FD/fdtd3d_0_base_module/fdtd3d_base_1_interface.hpp:50-112):
 * JSON with // comments, paths prefixed with proj_path.  rec_width is the
 * optional key of that name (0 when absent). */
typedef struct jv_argfile {
    char model_path[1024];
    char shot_path[1024];
    char rece_path[1024];
    char output_path[1024];
    int is_output, t_snap, pml_num;
    float fm, dt, T;
    int x_divide_num, y_divide_num, z_divide_num, slots_per_node;
    int rec_width;
    /* optional raw model (no reference key: the reference edits its model
     * loader to call Field::read_raw with a Frame, README.md:131-144):
     * vp/vs/rho files of n_rows*n_cols*n_slices float32, x fastest, prefixed
     * with proj_path; when vp_path is set, jv_open reads them instead of
     * model_path.  Empty / 0 when absent. */
    char vp_path[1024];
    char vs_path[1024];
    char rho_path[1024];
    int n_rows, n_cols, n_slices;
    float d_rows, d_cols, d_slices;
    int save_fld; /* optional key: jv_run_project also writes the images as .fld */
} jv_argfile;
jv_status jv_read_argfile(const char *proj_path, jv_argfile *out);

/* The reference's Frame as it lies in memory (the header of a .fld file):
 * .jarvis_0_meta/.jarvis_2_field/jarvis_0_frame_bones.hpp:9-51.  n_rows is
 * the x count (fastest), n_cols y, n_slices z; r = l + (n - 1) d; type is
 * Frame::Type (0 null, 1 vec, 2 mat, 3 cube, 10 line, 20 mesh, 30 grid). */
typedef struct jv_frame {
    uint64_t n_elem, n_rows, n_elem_slice;
    uint32_t n_cols, n_slices;
    float d_rows, d_cols, d_slices;
    float l_rows, l_cols, l_slices;
    float r_rows, r_cols, r_slices;
    int32_t type;
} jv_frame;
/* Fills *f as Frame(n_rows, n_cols, n_slices, d.., l..) does
 * (jarvis_0_frame_meat.hpp:27-65, set_frame_type :219-241). */
void jv_frame_make(uint64_t n_rows, uint32_t n_cols, uint32_t n_slices, float d_rows, float d_cols, float d_slices,
                   float l_rows, float l_cols, float l_slices, jv_frame *f);
/* Field::save(.., SaveFormat::binary_fld): path_noext + ".fld", the frame's
 * bytes then f->n_elem floats (jarvis_1_host_field_meat.hpp:81-89). */
jv_status jv_fld_write(const char *path_noext, const jv_frame *f, const float *data);
/* Field::load of a .fld file (jarvis_1_host_field_meat.hpp:41-64): the
 * frame into *f and, when data is not NULL, its n_elem floats (JV_EINVAL
 * if capacity, in floats, is smaller). */
jv_status jv_fld_read(const char *path, jv_frame *f, float *data, size_t capacity);
/* Field::read_raw (jarvis_1_host_field_meat.hpp:65-79): exactly n float32
 * values from a raw file (JV_EIO if its size differs). */
jv_status jv_raw_read(const char *path, size_t n, float *data);

/* Sets the survey: shot and receiver positions (x,y,z metres).  Only the
 * points inside gridphy are kept (SubGeometry::get_sub_shot_and_recv,
 * jarvis_device_geometry_meat.hpp:65-128).  Shots keep their input index. */
jv_status jv_set_geometry(jv_ctx *c, int n_shot, const float *shot_xyz, int n_recv, const float *recv_xyz);

/* Replaces the context's model with vp, vs, rho (host, gridphy, x fastest)
 * of the same grid: the extension into the absorbing layers and lambda, mu
 * are recomputed as jv_create does (elasticGeoModel<global>::initialize,
 * FD/fdtd3d_0_base_module/fdtd3d_base_3_geomodel_meat.hpp:405-489).  Device
 * buffers, tensor maps and captured time-loop graphs are kept, so a context
 * serves many models of one grid without being created again (the request
 * server's context pool does this).  The image stacks are not touched. */
jv_status jv_set_model(jv_ctx *c, const float *vp, const float *vs, const float *rho);

/* Sizes of the context's problem. */
typedef struct jv_info {
    jv_grid grid;
    int nt;
    int n_shot;          /* shots in the list (inside or not)        */
    int n_recv;          /* receivers kept (inside gridphy)          */
    int rec_width;
    int precision;
    long long n_ext;     /* cells of gridext                          */
    long long n_phy;     /* cells of gridphy                          */
    size_t store_bytes_per_step; /* VOWR bytes per time step          */
    size_t device_bytes; /* device memory held by the context         */
    int store_on_device; /* 1: boundary store in HBM, 0: pinned host  */
} jv_info;
jv_status jv_get_info(const jv_ctx *c, jv_info *info);

/* The options a context runs with: those it was created with, with the
 * kernel choice (kernel_variant, register budgets, planes per thread) as
 * made -- after kernel_variant -1, the measured one. */
jv_status jv_get_kernel_config(const jv_ctx *c, jv_options *out);

/* Reconstruction check of the last jv_rtm_shot (FP64, on the GPU): the energy
 * (sum of squares of the velocity and stress fields over gridphy) of the
 * source wavefield at the end of the forward pass, and of what is left of it
 * after the reverse loop has reconstructed it back to its zero initial
 * state.  Their ratio measures the VOWR reconstruction error (exact time
 * reversal at rec_width 4 up to FP32 rounding; an approximation below). */
jv_status jv_reconstruction_energy(const jv_ctx *c, double *e_forward_end, double *e_residual);

/* Forward modelling of one shot: replaces
 * fdtd3d_blend_elastic_model_mpi_module<pure_forward>::reset_for_next_shot
 * + mpi_sub_forward + SeisRecord::copy_seis_into_host
 * (FD/fdtd3d_3_model_mpi_blend/fdtd3d_blend_elastic_model_mpi_meat.hpp:38-88;
 *  FD/fdtd3d_0_base_module/fdtd3d_base_4_seisrecord_meat.hpp:312-321).
 * Outputs [n_recv][nt] (may be NULL to skip a component). */
jv_status jv_forward(jv_ctx *c, int shot, float *vx, float *vy, float *vz);
jv_status jv_forward_device(jv_ctx *c, int shot, float *d_vx, float *d_vy, float *d_vz);

/* Migrates one shot and stacks it into the context's images: replaces the
 * per-shot body of rtm3d_blend_model_mpi_module::mpi_sub_rtm3d
 * (RTM/rtm3d_1_model_mpi_blend/rtm3d_blend_elastic_model_mpi_meat.hpp:50-113):
 * forward with VOWR boundary store, then the fused time-reverse loop
 * (source reconstruction, receiver back-propagation, zero-lag imaging).
 * obs_*: the shot's observed traces [n_recv][nt]. */
jv_status jv_rtm_shot(jv_ctx *c, int shot, const float *obs_vx, const float *obs_vy, const float *obs_vz);
jv_status jv_rtm_shot_device(jv_ctx *c, int shot, const float *d_obs_vx, const float *d_obs_vy,
                             const float *d_obs_vz);

/* Migrates n shots (indices shots[0..n-1]) and stacks them, as the
 * per-shot loop of rtm3d_blend_model_mpi_module::mpi_sub_rtm3d does
 * (RTM/rtm3d_1_model_mpi_blend/rtm3d_blend_elastic_model_mpi_meat.hpp:50-113).
 * obs holds 3*n host pointers: vx, vy, vz of shot k at obs[3k..3k+2], each
 * [n_recv][nt] float32.  The copy of shot k+1's traces to the device runs
 * on a second stream while shot k's kernels run (page-locked host memory
 * lets the copies overlap).  jv_last_timing gives the summed device time
 * of the shots. */
jv_status jv_rtm_batch(jv_ctx *c, int n, const int *shots, const float *const *obs);

/* Image selectors. */
typedef enum jv_image_kind { JV_IMG_IP = 0, JV_IMG_PP = 1, JV_IMG_PS = 2, JV_IMG_SP = 3, JV_IMG_SS = 4 } jv_image_kind;

/* Zeroes the stacked images (MigImage::initialize). */
jv_status jv_image_reset(jv_ctx *c);
/* Copies one raw stacked accumulator (FP64, gridphy) to host memory. */
jv_status jv_image_get(jv_ctx *c, int kind, double *out);
/* The reference's final image step (rtm3d_blend_elastic_model_mpi_meat.hpp:
 * 123-124; RTM/rtm3d_0_image_module/rtm3d_iamge_kernel.hpp:118-135,184-200):
 * 7-point Laplacian of the UNcompensated pp/ps/sp/ss into lap (4 arrays of
 * gridphy, may be NULL), then source compensation I /= Ip where
 * Ip > 3.4e-38 into img (4 arrays: pp, ps, sp, ss; may be NULL).  Outputs are
 * float32 host arrays, as the reference saves them; the stacked
 * accumulators are not modified. */
jv_status jv_image_finalize(jv_ctx *c, float *img_pp, float *img_ps, float *img_sp, float *img_ss, float *lap_pp,
                            float *lap_ps, float *lap_sp, float *lap_ss);

/* Device-to-device copy of one raw stacked accumulator (FP64, gridphy) into
 * caller memory on the context's device, e.g. to reduce images of shot
 * replicas on several GPUs with a collective. */
jv_status jv_image_get_device(jv_ctx *c, int kind, double *d_out);

/* Overwrites one stacked accumulator (FP64, gridphy) from host memory
 * (jv_image_set) or from device memory on the context's device
 * (jv_image_set_device): loads the sum of the partial images of several
 * shot replicas (reduced by the caller, e.g. MPI_Allreduce or an NCCL
 * all-reduce) so that jv_image_finalize runs on the whole stack.  The
 * reference stacks every shot into one MigImage per process
 * (RTM/rtm3d_0_image_module/rtm3d_image_meat.hpp:74-96). */
jv_status jv_image_set(jv_ctx *c, int kind, const double *in);
jv_status jv_image_set_device(jv_ctx *c, int kind, const double *d_in);

/* Whole reference job: rtm3d_blend_model_mpi_module::mpi_sub_rtm3d
 * (RTM/rtm3d_1_model_mpi_blend/rtm3d_blend_elastic_model_mpi_meat.hpp:18-135):
 * model every shot and write {output_path}v?_seis_0_{shot}.txt, migrate every
 * shot, then write image_pp_0*.raw and image_pp_laplace_0*.raw with the
 * reference's names and formats.  Only for contexts made by jv_open. */
jv_status jv_run_project(jv_ctx *c);

/* In-place sum of n doubles over every rank of the caller's job (for
 * example MPI_Allreduce with MPI_IN_PLACE, or an NCCL all-reduce of a host
 * staging buffer); returns 0 on success. */
typedef int (*jv_reduce_fn)(double *buf, size_t n, void *user);

/* jv_run_project for a job of `world` processes (one GPU each), the
 * replacement of the reference's MPI job (rtm3d_blend_elastic_model_mpi_meat.hpp:
 * 18-135).  The reference splits the model into subdomains over its ranks;
 * here every rank holds the whole model and takes the shots s with
 * s % world == rank: it models them and writes their trace files,
 * migrates them, sums the five stacks over the job with `reduce` (called
 * five times, on every rank, in the same order), and rank 0 writes the
 * images.  world == 1 (reduce may be NULL) is jv_run_project. */
jv_status jv_run_project_shard(jv_ctx *c, int rank, int world, jv_reduce_fn reduce, void *user);

/* Jobs: forward modelling or migration of one shot, queued on the context
 * and run in submission order by a worker thread of the library, so that a
 * serving loop submits work and collects it later (jv_submit / jv_poll /
 * jv_wait / jv_cancel).  The reference has no queue: its driver runs the
 * shots of one job in a loop.  While jobs are queued or running, the other
 * calls that use the context return JV_ESTATE; the job calls are safe from
 * any thread.  Host buffers named in a job must stay valid until it ends. */
typedef enum jv_job_kind { JV_JOB_FORWARD = 0, JV_JOB_RTM = 1 } jv_job_kind;
typedef enum jv_job_state {
    JV_JOB_QUEUED = 0,
    JV_JOB_RUNNING = 1,
    JV_JOB_DONE = 2,
    JV_JOB_CANCELLED = 3
} jv_job_state;
typedef struct jv_job {
    int kind;            /* jv_job_kind                                              */
    int shot;            /* shot index of the context's geometry                     */
    const float *obs[3]; /* RTM: observed vx, vy, vz traces (host, [n_recv][nt]);
                            all NULL: the job models them on the device first         */
    float *out[3];       /* FORWARD: traces written here (host; NULL skips one)       */
} jv_job;
/* Queues a copy of *job; *id identifies it in the other job calls. */
jv_status jv_submit(jv_ctx *c, const jv_job *job, long long *id);
/* Non-blocking: *state (jv_job_state) and, once done, *result (may be NULL);
 * a failed job's message becomes jv_last_error(). */
jv_status jv_poll(jv_ctx *c, long long id, int *state, jv_status *result);
/* Waits for the job to end, at most timeout_s seconds (< 0: no limit);
 * returns JV_ETIMEOUT if it has not ended by then. */
jv_status jv_wait(jv_ctx *c, long long id, double timeout_s, jv_status *result);
/* Cancels a queued job (its result becomes JV_ECANCELED); a job that has
 * started runs to its end (JV_ESTATE). jv_close cancels the queued ones. */
jv_status jv_cancel(jv_ctx *c, long long id);

/* Requests and the server: a request is one shot of forward modelling or
 * RTM on a model and grid of its own.  jv_server keeps a queue and `slots`
 * worker threads; a worker takes the first queued request it can place --
 * on an idle pooled context of the same shape (grid, spacing, dt, fm, nt,
 * rec_width, precision, kind, receiver count), or on a new context whose
 * device footprint (jv_footprint) fits the memory still free under the
 * server's budget once idle pooled contexts are released, least recently
 * used first.  After the request the context stays pooled: the next request
 * of its shape only uploads its model (jv_set_model) and geometry.  So
 * requests of different sizes run concurrently on the GPU as slots and
 * memory come free.  A request's result does not depend on what else runs,
 * nor on whether its context was pooled.  The server answers poll/wait for
 * the latest 65536 ended requests; older ids are forgotten (JV_EINVAL).
 * The reference has no counterpart.  Host buffers named in a request must
 * stay valid until it ends. */
typedef struct jv_request {
    int kind;                   /* JV_JOB_FORWARD or JV_JOB_RTM                      */
    jv_grid grid;
    const float *vp, *vs, *rho; /* host, gridphy                                      */
    float dt, fm;
    int nt;
    int rec_width;              /* 0 -> 1                                            */
    float shot_xyz[3];          /* metres, inside gridphy                            */
    int n_recv;
    const float *recv_xyz;      /* metres; points outside gridphy are dropped        */
    const float *obs[3];        /* RTM: observed traces [n_kept][nt]; all NULL: the
                                   request models them first                          */
    float *out[3];              /* FORWARD: traces [n_kept][nt] (NULL skips one)     */
    double *image[5];           /* RTM: this shot's FP64 stacks ip, pp, ps, sp, ss
                                   (gridphy, NULL skips one)                         */
    int precision;              /* RTM boundary store: JV_FP32 (0), JV_BF16, JV_FP16; a
                                   16-bit store halves the store's share of the
                                   footprint the server admits the request by         */
} jv_request;
typedef struct jv_server jv_server;
typedef struct jv_server_stats {
    long long submitted, completed, failed, cancelled, running, queued;
    double p50_ms, p99_ms, mean_ms; /* submission to completion, over the latest 65536 completed */
    size_t bytes_in_use, budget;    /* running requests and pooled idle contexts */
    long long reused;               /* requests that ran on a pooled context      */
    long long pooled;               /* idle contexts pooled now                   */
    double device_ms;               /* device time of the completed requests'
                                       propagations (CUDA events on each
                                       context's stream, summed); with one slot,
                                       against the wall time, how busy the
                                       requests kept the GPU                     */
} jv_server_stats;
/* Device bytes a context holds for one request of this size with n_recv
 * receivers and an FP32 boundary store (an estimate from the layout; the
 * server's admission unit, which counts 2-byte records for a request with a
 * 16-bit store). */
jv_status jv_footprint(const jv_grid *grid, int nt, int rec_width, int kind, int n_recv, size_t *bytes);
/* hbm_budget 0: 90 % of the device's free memory now. */
jv_status jv_server_create(int device, int slots, size_t hbm_budget, jv_server **out);
/* JV_ENOMEM if the request alone exceeds the budget. */
jv_status jv_server_submit(jv_server *s, const jv_request *r, long long *id);
jv_status jv_server_poll(jv_server *s, long long id, int *state, jv_status *result);
jv_status jv_server_wait(jv_server *s, long long id, double timeout_s, jv_status *result);
jv_status jv_server_cancel(jv_server *s, long long id);
jv_status jv_server_get_stats(jv_server *s, jv_server_stats *out);
/* Cancels queued requests, waits for the running ones, frees the server. */
jv_status jv_server_close(jv_server *s);

/* Device time (ms) of the last jv_forward* / jv_rtm_shot* call, measured
 * with CUDA events around its kernels. */
jv_status jv_last_timing(const jv_ctx *c, double *ms);

/* The RTM shot in the phases of the reference's drivers, for callers that
 * drive the time loops themselves (the C++ front end jarvis_compat.hpp
 * runs the reference's rtm_forward / rtm_backward / rtm_reverse modules on
 * them).  jv_rtm_shot_device is
 *   jv_rtm_forward_pass(shot)                 fdtd3d_blend_elastic_model_mpi_module<rtm_forward>::
 *                                             mpi_sub_forward_for_restruct (FD/fdtd3d_3_model_mpi_blend/
 *                                             fdtd3d_blend_elastic_model_mpi_meat.hpp:125-155): modelling
 *                                             with the VOWR boundary store, graph-captured
 *   jv_rtm_reverse_begin(shot, d_obs)         rtm_backward / rtm_reverse reset_for_next_shot (:185-214):
 *                                             cleared receiver wavefield and shot image, the adjoint
 *                                             sources d_ox/d_oy/d_oz (device, [n_recv][nt])
 *   for it = nt-1 .. 0: jv_rtm_reverse_op     one kernel each, in the order of the reference's time-reverse
 *                                             loop (RTM/rtm3d_1_model_mpi_blend/
 *                                             rtm3d_blend_elastic_model_mpi_meat.hpp:64-113)
 *   jv_rtm_reverse_end                        the shot image added to the FP64 stacks, the reconstruction
 *                                             check (jv_reconstruction_energy)
 * The per-op path launches kernels one at a time (no graphs), so it is
 * slower than jv_rtm_shot_device; the results are the same, bit for bit.
 * Time indices: `it` is the time step of the loop; for the two boundary
 * replays it is the index of the record replayed (the reference passes
 * it - 1; records outside 0..nt-2 replay nothing). */
typedef enum jv_rtm_op {
    JV_OP_INJECT_RECEIVERS = 0,       /* adjoint sources at it (sub_rtm_reverse_add_vel_source)       */
    JV_OP_BACKWARD_STRESS = 1,        /* source wavefield, stress backward in time, its source
                                         subtracted at it (cuda_subtract_stress_source fused)         */
    JV_OP_REVERSE_VEL_PML = 2,        /* receiver wavefield, absorbing layers of the velocity update  */
    JV_OP_REVERSE_VEL = 3,            /* receiver wavefield, velocity update of gridphy               */
    JV_OP_INJECT_BOUNDARY_STRESS = 4, /* stored stress boundary layers of record it                   */
    JV_OP_BACKWARD_VEL_IMAGE = 5,     /* source wavefield, velocity backward in time, with the
                                         zero-lag imaging condition fused (cal_correlation_from_wave) */
    JV_OP_REVERSE_STRESS_PML = 6,     /* receiver wavefield, absorbing layers of the stress update
                                         (nothing where they run inside JV_OP_REVERSE_STRESS)          */
    JV_OP_REVERSE_STRESS = 7,         /* receiver wavefield, stress update                            */
    JV_OP_INJECT_BOUNDARY_VEL = 8     /* stored velocity boundary layers of record it                 */
} jv_rtm_op;
jv_status jv_rtm_forward_pass(jv_ctx *c, int shot);
jv_status jv_rtm_reverse_begin(jv_ctx *c, int shot, const float *d_ox, const float *d_oy, const float *d_oz);
jv_status jv_rtm_reverse_op(jv_ctx *c, int op, int it);
jv_status jv_rtm_reverse_end(jv_ctx *c);

/* Per-kernel timing: with profiling on, the time loops launch kernels
 * directly (no graphs) and bracket each launch with CUDA events on the
 * context's stream; jv_profile_entry returns, for entry idx, the kernel
 * name, the summed device time and the launch count since profiling was
 * switched on (JV_EINVAL past the last entry).  The reference prints
 * per-shot times only (cuda_tic/cuda_toc, .jarvis_0_meta/.jarvis_0_math/
 * jarvis_2_device_math_bones.hpp:26-38). */
jv_status jv_set_profiling(jv_ctx *c, int on);
jv_status jv_profile_entry(const jv_ctx *c, int idx, const char **name, double *total_ms, long long *launches);

/* Forward modelling of one shot that allocates no device memory, for
 * callers that cannot call cudaMalloc/cudaFree when they model (their
 * memory pool already holds the free device memory, or an allocation could
 * block or synchronise a latency-critical path).  No counterpart in the
 * reference.  Inputs are device arrays on gridphy (vp, vs, rho) and host
 * positions; d_vx/d_vy/d_vz receive [n_kept][nt] traces of the receivers
 * inside gridphy (*n_kept of them, at most n_recv).  Working memory comes
 * from one 64 MiB array compiled into the library, held on every device that
 * loads it; problems that need more are rejected with JV_EINVAL (the
 * limit is about 0.5 M cells of gridext, e.g. a 60^3 interior with a 10-cell
 * absorbing layer).  The first call on a device (and again after the
 * device's context was replaced, e.g. by cudaDeviceReset) sets up: it looks
 * up that array's address and uploads the constant finite-difference
 * coefficients, which synchronises the device, so make that first call
 * before any stream capture.  All calls share the array: calls whose GPU
 * work overlaps race; the call clears what must start at zero and returns
 * after its work on `stream` (cudaStream_t, NULL for the legacy stream) has
 * finished, on failure as well. */
jv_status jv_forward_noalloc(const jv_grid *grid, const float *d_vp, const float *d_vs, const float *d_rho, float dt,
                             float fm, int nt, const float *src_xyz, int n_recv, const float *recv_xyz, float *d_vx,
                             float *d_vy, float *d_vz, int *n_kept, void *stream);

/* Attainable HBM bandwidth of a pointwise pass that reads n_read and writes
 * n_write arrays of n floats each (n a multiple of 4; one float4 of every
 * array per thread, every load issued before the stores), in GB/s of bytes
 * moved, from the median device time of `reps` launches after one warm-up.
 * The supported (n_read, n_write) pairs are the footprints of this
 * library's kernels and a copy: (1,1) (2,1) (10,3) (12,7) (14,6) (25,11).
 * Allocates its arrays on `device` and frees them before it returns.  A
 * diagnostic for the roofline of many-array kernels; no counterpart in the
 * reference. */
jv_status jv_stream_probe(int device, int n_read, int n_write, size_t n, int reps, double *gbs);

/* Waits for all work of the context. */
jv_status jv_sync(jv_ctx *c);

jv_status jv_close(jv_ctx *c);

/* Message of the last failed call on this thread ("" if none). */
const char *jv_last_error(void);

/* Library / kernel build facts, for diagnostics. */
const char *jv_build_info(void);

#ifdef __cplusplus
}
#endif
#endif /* JV_JV_H */
