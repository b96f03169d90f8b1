// engine.hpp -- one modelling/RTM problem resident on one GPU.
//
// The Engine owns every device buffer of a problem (model, two wavefields,
// CPML memory variables, VOWR boundary store, traces, FP64 images) and runs
// the time loops of the reference's blend modules with the kernels of
// kernels.cu, replaying each chunk of time steps as one CUDA graph.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "jv/jv.h"
#include "jv_internal.hpp"

namespace jv {

// Staggered-grid Taylor coefficients of half-order `order`
// (src/jarvis_cpp/jarvis/.jarvis_1_util/.jarvis_2_geometry/
// jarvis_device_geometry_bones.hpp:29-49).
void diff_coeff(int order, double *c);
// get_gap_num (.jarvis_0_meta/.jarvis_2_field/jarvis_3_device_field_meat.hpp:9-22)
int gap_num(float l, float r, float d);
// ntime = ceil(T/dt) in float (FD/fdtd3d_0_base_module/fdtd3d_base_4_seisrecord_meat.hpp:278)
int ntime(float T, float dt);
// Ricker wavelet as the reference builds it (seisrecord_meat.hpp:279-285)
void ricker(int nt, float fm, float dt, float *w);

// message returned by jv_last_error() on the calling thread
void set_last_error(const std::string &m);

// RTM of `shot` on traces the context models first (forward modelling of
// the same shot); the traces stay in the context's device buffer (the
// request server's RTM requests without observed traces)
jv_status rtm_self_modelled(jv_ctx *c, int shot);

// Pitched gridext layout of a gridphy + pml problem (elem = base + xoff +
// i + sy*j + sz*k, first gridphy column 128-byte aligned); *field_elems =
// floats of one field array (gridext plus tail slack for the aligned
// x groups of the absorbing-layer kernels).
GridDev make_layout(const jv_grid &grid, size_t *field_elems);
// The six CPML slabs (FD/fdtd3d_0_base_module/fdtd3d_base_6_pml_meat.hpp:29-94)
// with their launch shapes and memory-variable arena offsets; *psi_total =
// floats of one wavefield's memory-variable arena.  dt, ax and psi are
// left for the caller.
CpmlDev make_pml_slabs(const GridDev &g, int zp, long long *psi_total);
// Per-axis damping factor tables {K, K_half, alpha, alpha_half}, K = 0
// outside the axis' absorbing range
// (FD/fdtd3d_1_cpml_mpi_module/fdtd3d_cpml_mpi_1_host_meat.hpp:147-620).
void pml_axis_tables(const GridDev &g, float fm, std::vector<float4> t[3]);
// VOWR face boxes of rec_width r for a layout, velocity fields first;
// *per_step = values of one step's record, *blocks = 256-thread blocks.
// With vec (the FP32 store) box offsets are rounded up to 4 values and a
// box whose rows are 4-aligned whole x groups moves 4 values a thread.
std::vector<SegDev> vowr_segments(const GridDev &g, int r, long long *per_step, long long *blocks, bool vec);
// Device bytes a context of this problem holds after one forward (rtm false)
// or RTM shot (rtm true) with a boundary store of `precision`
// (jv_precision), traces excluded.
size_t footprint_bytes(const jv_grid &grid, int nt, int rec_width, bool rtm, int precision);
// Uploads the staggered coefficient rows of every order and the 4th-order
// CPML pair to constant memory of the current device.
int upload_all_coefficients();

struct Status {
    jv_status code = JV_OK;
    std::string msg;
    explicit operator bool() const { return code == JV_OK; }
};

class Engine {
   public:
    ~Engine();
    static Status create(const jv_grid &grid, const float *vp, const float *vs, const float *rho, float dt, float fm,
                         int nt, const jv_options &opt, Engine **out);

    Status set_geometry(int n_shot, const float *shot_xyz, int n_recv, const float *recv_xyz);
    // a new model of the same grid (host arrays on gridphy); buffers, tensor
    // maps and captured graphs stay as they are
    Status set_model(const float *vp, const float *vs, const float *rho);
    Status forward(int shot, float *d_vx, float *d_vy, float *d_vz);
    // obs_ready: an event the observed traces' copy records; the reverse
    // loop, the first user of the traces, waits for it, so the copy runs
    // beside the forward pass
    Status rtm_shot(int shot, const float *d_ox, const float *d_oy, const float *d_oz,
                    cudaEvent_t obs_ready = nullptr);
    // the phases of rtm_shot, for drivers that run them one by one: the
    // forward pass with the boundary store, the opening of the time-reverse
    // loop, one of its kernels (jv_rtm_op) at a time index, and its end
    // (reconstruction check, the shot image added to the stacks)
    Status rtm_forward_pass(int shot);
    Status rtm_reverse_begin(int shot, const float *d_ox, const float *d_oy, const float *d_oz);
    Status rtm_reverse_op(int op, int it);
    Status rtm_reverse_end();
    Status image_reset();
    Status image_get(int kind, double *host_out);
    Status image_finalize(float *host_out[8]);
    Status image_get_device(int kind, double *dev_out);
    Status image_set(int kind, const double *src, bool src_on_device);

    // per-kernel timing with CUDA events (direct launches, no graphs)
    void set_profiling(bool on);
    int profile_count() const { return (int)prof_names_.size(); }
    bool profile_entry(int i, const char **name, double *ms, long long *launches) const;
    Status sync();
    void info(jv_info *i) const;
    double last_ms() const { return last_ms_; }
    void set_last_ms(double ms) { last_ms_ = ms; }
    int nrec() const { return nrec_; }
    int nt() const { return nt_; }
    cudaStream_t stream() const { return stream_; }
    int device() const { return dev_; }

    // project bookkeeping (jv_open)
    std::string output_path;

   private:
    Engine() = default;
    Status alloc_all(const float *vp, const float *vs, const float *rho);
    Status upload_model(const float *vp, const float *vs, const float *rho);
    Status check_shot(int shot, long long *src) const;
    Status run_loop(int kind, int nsteps);
    Status launch_step(int kind, int off, bool advance);
    Status autotune(bool neutral);

  public:
    // the options this context runs with, the kernel choice as made
    void kernel_config(jv_options *o) const {
        *o = opt_;
        o->kernel_variant = kc_.variant;
        o->min_blocks = kc_.minb;
        o->pml_min_blocks = kc_.pml_minb;
        o->planes_per_thread = kc_.zp;
        o->pml_planes_per_thread = kc_.pml_zp;
        o->run_chunks = use_full_ ? fullF_.geo.Q : 0;
        o->tile_gx = kc_.gx;
        o->tile_gy = kc_.gy;
    }

  private:
    Status cu(cudaError_t e, const char *what) const;
    Status zero_wave(const WaveDev &w, int nfld);
    Status zero_psi(const CpmlDev &c);
    Status set_state(int it, long long src, float *const tr[3], const float *const obs[3]);
    Status rtm_prepare();
    Status reverse_end_launch();
    StepState h_state_{};   // host copy of the last step state written
    int fwd_shot_ = -1;     // shot of the last RTM forward pass
    bool rev_open_ = false;  // a time-reverse loop is open

    jv_grid grid_{};
    jv_options opt_{};
    float dt_ = 0.f, fm_ = 0.f;
    int nt_ = 0;
    int dev_ = 0;
    cudaStream_t stream_ = nullptr;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    double last_ms_ = 0.0;

    GridDev g_{};
    KCfg kc_{};
    WaveMaps mapsF_{}, mapsR_{};  // TMA descriptors of the velocity fields (variant 3)
    FullMaps fullF_{}, fullR_{};  // TMA descriptors of the full-gridext stress kernel (variant 4)
    float *fzpsiF_ = nullptr, *fzpsiR_ = nullptr;  // its axis-major stress memory variables
    long long fz_psi_total_ = 0;                   // floats of one of them
    double *energy_d_ = nullptr;          // device: the two energies of the reconstruction check
    double recon_energy_[2] = {0.0, 0.0};  // host copy after each RTM shot

  public:
    // FP64 energy of the source wavefield over gridphy at the end of the last
    // RTM shot's forward pass, and after its reconstruction back to t = 0
    void reconstruction_energy(double *fwd, double *res) const {
        *fwd = recon_energy_[0];
        *res = recon_energy_[1];
    }

  private:
    bool use_full_ = false;                        // the stress update of absorbing steps runs in stress_fz
    bool vel_full_ = false;                        // the forward passes' velocity update runs in vel_fz
    int *zm_err_ = nullptr;       // device flag of variant 3's bounded waits
    Status check_zm_err();
    size_t field_elems_ = 0;  // elements per pitched field
    std::vector<void *> allocs_;
    size_t dev_bytes_ = 0;

    float *vp_ = nullptr, *bdt_ = nullptr, *lam_ = nullptr, *mu_ = nullptr;  // bdt_: dt / rho
    WaveDev F_{}, R_{};
    CpmlDev cpF_{}, cpR_{};
    CpmlDev cpml_proto_{};     // slab table shared by both wavefields
    long long psi_total_ = 0;  // memory-variable floats per wavefield
    float4 *axis_d_[3] = {nullptr, nullptr, nullptr};
    CpmlDev make_cpml(float *psi) const;
    float *wavelet_ = nullptr;
    StepState *st_ = nullptr;

    // geometry
    std::vector<float> shots_;      // all shots (x,y,z)
    std::vector<long long> rec_h_;  // element index of kept receivers
    long long *rec_d_ = nullptr;
    int nrec_ = 0;
    int nshot_ = 0;

    // VOWR store
    std::vector<SegDev> segs_h_;
    VowrDev vowr_{};
    long long per_step_ = 0;
    float *store_ = nullptr;
    void *host_store_ = nullptr;   // pinned, mapped host memory of a host-resident store
    bool store_on_host_ = false;
    int nslot_ = 0;

    StackDev img_{};             // FP64 stacks over shots
    ImageDev shot_img_{};        // FP32 image of the shot being migrated
    size_t shot_img_pitch_ = 0;  // floats between its five arrays
    float *fin_ = nullptr;  // 8 * n_phy finalize buffer

    // graphs: key = kind * 100000 + steps
    std::map<long long, cudaGraphExec_t> graphs_;

    Status alloc(void **p, size_t bytes);

    // profiling state
    bool prof_ = false;
    std::vector<std::string> prof_names_;
    std::vector<double> prof_ms_;
    std::vector<long long> prof_n_;
    struct ProfRec { int id; cudaEvent_t a, b; };
    std::vector<ProfRec> prof_pending_;
    std::vector<cudaEvent_t> prof_pool_;
    size_t prof_used_ = 0;
    int prof_id(const char *name);
    cudaEvent_t prof_event();
    Status prof_collect();

    // JV_CHECK_FINITE=1: after every launch, count non-finite values of
    // both wavefields and the image stacks (direct launches, no graphs)
    bool check_finite_ = false;
    unsigned long long *nf_ = nullptr;
    int cur_kind_ = -1;
    Status check_finite(const char *after);
};

// kinds of time-loop steps
enum StepKind : int { kStepModel = 0, kStepRtmFwd = 1, kStepRtmRev = 2 };

}  // namespace jv
