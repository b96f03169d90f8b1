/*
 * jv_oracle.h -- CPU restatement of the jarvis elastic FDTD modelling and
 * VOWR reverse-time-migration path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * product (libjv.so): only tests/, __graft_entry__.smoke() and the CPU
 * baseline legs of bench.py load it.  The product never links or calls it.
 *
 * Compiled twice from one source: JVO_REAL=double (the FP64 oracle,
 * liboracle_f64.so) and JVO_REAL=float (an FP32 restatement,
 * liboracle_f32.so, used to separate discretisation error from FP32 error).
 *
 * Every routine names the reference file:line it restates (paths relative
 * to the reference project root; FD = src/jarvis_cpp/jarvis/.jarvis_2_app/
 * .jarvis_3_seismology/elastic_1_fdtd3d_model_mpi, RTM = the sibling
 * elastic_1_rtm3d_model_mpi directory).
 */
#ifndef JV_ORACLE_H
#define JV_ORACLE_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

/* One modelling / migration problem.  Grid sizes are the PHYSICAL grid
 * (gridphy); the extended grid adds `pml` cells on each of the six faces
 * (FD/fdtd3d_0_base_module/fdtd3d_base_3_geomodel_meat.hpp:405-453). */
typedef struct jvo_problem {
    int nx, ny, nz;        /* gridphy cells, x fastest                    */
    int pml;               /* argfile pml_num = margin on every face      */
    float dx, dy, dz;      /* spacing [m]                                  */
    float dt, fm, T;       /* argfile dt, fm, T                            */
    int rec_width;         /* GeoConst::rec_width (VOWR)                   */
    int n_shot;            /* all shots of shot.txt (x,y,z metres)         */
    const float *shot_xyz;
    int n_recv;            /* receivers of rece.txt (x,y,z metres)        */
    const float *recv_xyz;
    int nthreads;          /* OpenMP threads (0 = runtime default)         */
} jvo_problem;

/* ntime = ceil(T/dt) evaluated in float
 * (FD/fdtd3d_0_base_module/fdtd3d_base_4_seisrecord_meat.hpp:278). */
int jvo_ntime(float T, float dt);

/* Staggered-grid Taylor coefficients of half-order `order`
 * (src/jarvis_cpp/jarvis/.jarvis_1_util/.jarvis_2_geometry/
 * jarvis_device_geometry_bones.hpp:29-49). */
void jvo_diff_coeff(int order, double *c);

/* Ricker wavelet, rounded to float as the reference stores it
 * (FD/fdtd3d_0_base_module/fdtd3d_base_4_seisrecord_meat.hpp:273-285). */
void jvo_ricker(int nt, float fm, float dt, float *w);

/* Reference get_gap_num (.jarvis_0_meta/.jarvis_2_field/
 * jarvis_3_device_field_meat.hpp:9-22). */
int jvo_gap_num(float l, float r, float d);

/* CPML coefficients of one axis at extended index `c` of an axis of `n`
 * extended cells, margin `m`, local vp (FD/fdtd3d_1_cpml_mpi_module/
 * fdtd3d_cpml_mpi_1_host_meat.hpp:147-620).  Returns 0 and a=0,b=1 outside
 * the PML of that axis.  out = {a, b, a_half, b_half}. */
int jvo_cpml_ab(int c, int n, int m, float vp, float delta, float fm,
                float dt, double *out);

/* Receivers / shots that fall inside gridphy, in file order
 * (src/jarvis_cpp/jarvis/.jarvis_1_util/.jarvis_2_geometry/
 * jarvis_device_geometry_meat.hpp:65-128).  Returns the count and, when
 * idx != NULL, their indices into the input list. */
int jvo_select_inside(const jvo_problem *p, const float *xyz, int n, int *idx);

/* Forward modelling of shot `shot` (pure_forward,
 * FD/fdtd3d_3_model_mpi_blend/fdtd3d_blend_elastic_model_mpi_meat.hpp:44-88).
 * vp/vs/rho: gridphy float arrays.  traces: [n_sel_recv][nt] per component
 * (time fastest, FD/fdtd3d_0_base_module/fdtd3d_base_4_seisrecord_meat.hpp:
 * 57-77).  Returns 0 on success. */
int jvo_forward(const jvo_problem *p, const float *vp, const float *vs,
                const float *rho, int shot, double *tr_vx, double *tr_vy,
                double *tr_vz);

/* RTM of one shot (RTM/rtm3d_1_model_mpi_blend/
 * rtm3d_blend_elastic_model_mpi_meat.hpp:50-113): forward with boundary
 * store, then the fused time-reverse loop.  obs_*: the shot's traces
 * [n_sel_recv][nt].  Image accumulators (gridphy, FP64) are ADDED to, so
 * shots stack: ip = source illumination Ip_fd, then pp, ps, sp, ss.
 * When recon_err != NULL it receives the relative L2 difference between
 * the reconstructed source wavefield (vx,vy,vz over gridphy) at it == 0
 * and the forward wavefield after step 0. */
int jvo_rtm_shot(const jvo_problem *p, const float *vp, const float *vs,
                 const float *rho, int shot, const double *obs_vx,
                 const double *obs_vy, const double *obs_vz, double *ip,
                 double *pp, double *ps, double *sp, double *ss,
                 double *recon_err);

/* Final image processing (RTM/rtm3d_1_model_mpi_blend/
 * rtm3d_blend_elastic_model_mpi_meat.hpp:123-124): 7-point Laplacian of the
 * UNcompensated images into lap_* (zero outside cells 2..n-3), then
 * in-place source compensation I /= Ip where Ip > 3.4e-38. */
void jvo_finalize_image(int nx, int ny, int nz, const double *ip,
                        double *pp, double *ps, double *sp, double *ss,
                        double *lap_pp, double *lap_ps, double *lap_sp,
                        double *lap_ss);

/* Bounded work sample for the CPU baseline: `steps` time steps of each
 * propagation of one RTM shot (forward with boundary store, and the
 * reverse loop with reconstruction, receiver propagation and imaging) on
 * the full grid.  Returns the cell-updates done (steps * (2 N_ext + N_phy)). */
double jvo_rtm_sample(const jvo_problem *p, const float *vp, const float *vs,
                      const float *rho, int shot, int steps);

/* Storage-precision study (not part of the reference's algorithm; default
 * off): with mode 1 (FP16) or 2 (BF16) every later call rounds each stored
 * wavefield component to 16 bits after every update that writes it, with
 * one power-of-two FP32 scale per z plane of gridext (FP16: the plane's
 * largest magnitude maps into (2^11, 2^12]); mode 0 restores plain
 * storage.  Arithmetic stays JVO_REAL.  Used to measure what 16-bit
 * wavefield storage would cost in trace and image error. */
void jvo_set_store16(int mode);

#ifdef __cplusplus
}
#endif
#endif
