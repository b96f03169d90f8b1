/*
 * jarvis_compat.hpp -- the driver-facing C++ names of the jarvis elastic
 * RTM job, implemented over libjv's C ABI (jv/jv.h), so that a driver
 * written against the reference's classes builds against libjv.
 *
 * What a reference driver calls, and what it becomes here
 * (RTM = src/jarvis_cpp/jarvis/.jarvis_2_app/.jarvis_3_seismology/elastic_1_rtm3d_model_mpi,
 *  FD  = src/jarvis_cpp/jarvis/.jarvis_2_app/.jarvis_3_seismology/elastic_1_fdtd3d_model_mpi):
 *
 *   jarvis_mpi_init / jarvis_mpi_final        MPI_Init/Finalize when JV_COMPAT_MPI is defined,
 *                                             else one process (rank 0 of 1)
 *   ArgList::mpi_read_arg_file                jv_read_argfile
 *                                             (FD/fdtd3d_0_base_module/fdtd3d_base_1_interface.hpp:27-113)
 *   jarvis_global_mpicu_Stream_t::initialize  records the split; the reference builds
 *                                             subdomain streams and halo requests here
 *   rtm3d_blend_model_mpi_module::link        keeps the ArgList
 *   rtm3d_blend_model_mpi_module::mpi_sub_rtm3d
 *                                             jv_open + jv_run_project_shard over the
 *                                             job's ranks (RTM/rtm3d_1_model_mpi_blend/
 *                                             rtm3d_blend_elastic_model_mpi_bones.hpp:6-19)
 *   device_mpi_sub_rtm3d                      the same (RTM/rtm3d_2_model_mpi_blend_test/
 *                                             rtm3d_blend_elastic_model_mpi_device.cu:8-11)
 *   fdtd3d_blend_elastic_model_mpi_module<SimulateType::pure_forward>
 *                                             link / initialize / mpi_sub_forward /
 *                                             reset_for_next_shot over jv_forward, traces
 *                                             kept in host vectors
 *                                             (FD/fdtd3d_3_model_mpi_blend/
 *                                             fdtd3d_blend_elastic_model_mpi_bones.hpp:18-31)
 *
 * Differences a driver sees: x/y/z_divide_num must be 1 (every rank holds
 * the whole model; with several ranks each takes its share of the shots
 * and the stacks are summed with MPI_Allreduce); failures print the
 * library's message and call std::abort(), as the reference does.
 * GPU_NUM_PER_NODE defaults to 8, the GPUs of a B200 node.
 */
#ifndef JV_JARVIS_COMPAT_HPP
#define JV_JARVIS_COMPAT_HPP

#include <cuda_runtime_api.h>

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "jv/jv.h"

#ifdef JV_COMPAT_MPI
#include <mpi.h>
#endif

#ifndef GPU_NUM_PER_NODE
#define GPU_NUM_PER_NODE 8
#endif

namespace jarvis {

// ---------------------------------------------------------------- process
#ifdef JV_COMPAT_MPI
#define jarvis_mpi_init(argc, argv, mpi_rank, mpi_size) \
    MPI_Init(&(argc), &(argv));                         \
    int mpi_rank = 0, mpi_size = 1;                     \
    MPI_Comm_rank(MPI_COMM_WORLD, &mpi_rank);           \
    MPI_Comm_size(MPI_COMM_WORLD, &mpi_size)
#define jarvis_mpi_final MPI_Finalize()
#else
// one process: the MPI calls a reference driver makes become no-ops
#define jarvis_mpi_init(argc, argv, mpi_rank, mpi_size) \
    int mpi_rank = 0, mpi_size = 1;                     \
    (void)(argc);                                       \
    (void)(argv)
#define jarvis_mpi_final ((void)0)
#ifndef MPI_COMM_WORLD
#define MPI_COMM_WORLD 0
#endif
inline int MPI_Barrier(int) { return 0; }
#endif

inline void jv_compat_die(const char *what) {
    std::fprintf(stderr, "[jv] %s: %s\n", what, jv_last_error());
    std::abort();
}

inline void jv_compat_cuda_check(cudaError_t e, const char *file, int line) {
    if (e != cudaSuccess) {
        std::fprintf(stderr, "[jv] CUDA error %s at %s:%d\n", cudaGetErrorString(e), file, line);
        std::abort();
    }
}
#define jarvis_handle_cuda_error(err) (::jarvis::jv_compat_cuda_check((err), __FILE__, __LINE__))

// free/total device memory of one GPU, printed
inline void jarvis_get_gpu_memory(int i_device) {
    size_t fr = 0, tot = 0;
    cudaSetDevice(i_device);
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess)
        std::printf("[GPU %d] free %.2f GB of %.2f GB\n", i_device, fr / 1e9, tot / 1e9);
}

// ---------------------------------------------------------------- config
enum class SimulateType { pure_forward, rtm_forward, rtm_backward, rtm_reverse, fwi };

struct ArgList {
    std::string proj_path, model_path, shot_path, recv_path, output_path;
    int mpi_rank = 0, mpi_size = 1;
    int x_divide_num = 1, y_divide_num = 1, z_divide_num = 1, slots_per_node = 1;
    int pml_num = 0, t_snap = -1;
    float fm = 0.f, T = 0.f, dt = 0.f;
    bool is_output = false;

    void mpi_read_arg_file(std::string _proj_path, int _mpi_rank, int _mpi_size) {
        jv_argfile a;
        if (jv_read_argfile(_proj_path.c_str(), &a) != JV_OK) jv_compat_die("argfile");
        proj_path = _proj_path;
        mpi_rank = _mpi_rank;
        mpi_size = _mpi_size;
        model_path = a.model_path;
        shot_path = a.shot_path;
        recv_path = a.rece_path;
        output_path = a.output_path;
        x_divide_num = a.x_divide_num;
        y_divide_num = a.y_divide_num;
        z_divide_num = a.z_divide_num;
        slots_per_node = a.slots_per_node;
        pml_num = a.pml_num;
        t_snap = a.t_snap;
        fm = a.fm;
        T = a.T;
        dt = a.dt;
        is_output = a.is_output != 0;
    }
};

// The reference's per-rank stream/communicator set.  Nothing of it is
// needed here: libjv keeps one stream per context.
struct jarvis_global_mpicu_Stream_t {
    int x_divide_num = 1, y_divide_num = 1, z_divide_num = 1, mpi_rank = 0, mpi_size = 1, slots_per_node = 1;
    void initialize(int x, int y, int z, int rank, int size, int slots) {
        x_divide_num = x; y_divide_num = y; z_divide_num = z;
        mpi_rank = rank; mpi_size = size; slots_per_node = slots;
    }
    void clear() {}
};

// ---------------------------------------------------------------- jobs
namespace jv_compat_detail {
inline jv_ctx *open(const ArgList &a) {
    if (a.x_divide_num * a.y_divide_num * a.z_divide_num != 1)
        std::fprintf(stderr, "[jv] x/y/z_divide_num must be 1: every rank holds the whole model\n");
    jv_options o;
    jv_options_default(&o);
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) o.device = dev;
    jv_ctx *c = nullptr;
    if (jv_open(a.proj_path.c_str(), &o, &c) != JV_OK) jv_compat_die("jv_open");
    return c;
}
#ifdef JV_COMPAT_MPI
inline int allreduce(double *buf, size_t n, void *) {
    return MPI_Allreduce(MPI_IN_PLACE, buf, (int)n, MPI_DOUBLE, MPI_SUM, MPI_COMM_WORLD) == MPI_SUCCESS ? 0 : 1;
}
#endif
}  // namespace jv_compat_detail

class rtm3d_blend_model_mpi_module {
   public:
    ArgList *arg_list_p = nullptr;
    jarvis_global_mpicu_Stream_t *jarvis_mpi_cuda_stream_p = nullptr;

    void link(ArgList *_arg_list_p, jarvis_global_mpicu_Stream_t *_stream_p) {
        arg_list_p = _arg_list_p;
        jarvis_mpi_cuda_stream_p = _stream_p;
    }
    // the whole job: model and save every shot's traces, migrate, stack
    // over ranks, Laplacian + compensation, save the images
    void mpi_sub_rtm3d() {
        if (!arg_list_p) jv_compat_die("mpi_sub_rtm3d before link");
        jv_ctx *c = jv_compat_detail::open(*arg_list_p);
        const int rank = arg_list_p->mpi_rank, world = arg_list_p->mpi_size;
        jv_reduce_fn red = nullptr;
#ifdef JV_COMPAT_MPI
        red = &jv_compat_detail::allreduce;
#else
        if (world != 1) jv_compat_die("several ranks need JV_COMPAT_MPI");
#endif
        if (jv_run_project_shard(c, rank, world, red, nullptr) != JV_OK) jv_compat_die("mpi_sub_rtm3d");
        jv_close(c);
    }
};

inline void device_mpi_sub_rtm3d(rtm3d_blend_model_mpi_module *rtm_mpi) { rtm_mpi->mpi_sub_rtm3d(); }

template <SimulateType simulate_type>
class fdtd3d_blend_elastic_model_mpi_module;

// Forward modelling of one shot at a time; the traces of the last shot are
// kept in vx_seis / vy_seis / vz_seis ([n_recv][nt], time fastest).
template <>
class fdtd3d_blend_elastic_model_mpi_module<SimulateType::pure_forward> {
   public:
    ArgList *arg_list_p = nullptr;
    std::vector<float> vx_seis, vy_seis, vz_seis;
    int n_recv = 0, nt = 0, n_shot = 0;

    ~fdtd3d_blend_elastic_model_mpi_module() {
        if (ctx_) jv_close(ctx_);
    }
    void link(ArgList *_arg_list_p) { arg_list_p = _arg_list_p; }
    void initialize() {
        if (!arg_list_p) jv_compat_die("initialize before link");
        ctx_ = jv_compat_detail::open(*arg_list_p);
        jv_info i;
        jv_get_info(ctx_, &i);
        n_recv = i.n_recv;
        nt = i.nt;
        n_shot = i.n_shot;
        const size_t per = (size_t)n_recv * nt;
        vx_seis.assign(per, 0.f);
        vy_seis.assign(per, 0.f);
        vz_seis.assign(per, 0.f);
    }
    void mpi_sub_forward(int _i_shot) {
        if (!ctx_) jv_compat_die("mpi_sub_forward before initialize");
        if (jv_forward(ctx_, _i_shot, vx_seis.data(), vy_seis.data(), vz_seis.data()) != JV_OK)
            jv_compat_die("mpi_sub_forward");
    }
    // every shot starts from a zero wavefield in libjv; nothing to reset
    void reset_for_next_shot() {}

   private:
    jv_ctx *ctx_ = nullptr;
};

}  // namespace jarvis

#endif /* JV_JARVIS_COMPAT_HPP */
