/*
 * jarvis_compat.hpp -- the driver-facing C++ names of the jarvis elastic
 * modelling and RTM modules, implemented over libjv's C ABI (jv/jv.h), so
 * that a driver written against the reference's classes builds against
 * libjv.  Header only; link with -ljv -lcudart.
 *
 * What a reference driver calls, and what it becomes here
 * (RTM  = src/jarvis_cpp/jarvis/.jarvis_2_app/.jarvis_3_seismology/elastic_1_rtm3d_model_mpi,
 *  FD   = src/jarvis_cpp/jarvis/.jarvis_2_app/.jarvis_3_seismology/elastic_1_fdtd3d_model_mpi,
 *  META = src/jarvis_cpp/jarvis/.jarvis_0_meta):
 *
 *   GeoConst / geo_const                   the compile-time orders (FD/fdtd3d_0_base_module/
 *                                          fdtd3d_base_1_interface.hpp:10-16); rec_width is
 *                                          JV_COMPAT_REC_WIDTH (default 1), passed to every context
 *   Frame                                  META/.jarvis_2_field/jarvis_0_frame_bones.hpp:9-51, the
 *                                          same members and layout (a .fld header)
 *   Field<T, MemType, MemBlock::single>    META/.jarvis_2_field/jarvis_1_host_field_bones.hpp,
 *                                          jarvis_3_device_field_bones.hpp:22-153: host and/or device
 *                                          buffers on a Frame, read_raw / load / save / cu_save in the
 *                                          reference's formats.  MemBlock::multiple / puppet (the CMM
 *                                          blocks of the halo exchange) are not provided: the whole
 *                                          model is resident on one GPU
 *   ArgList::mpi_read_arg_file             jv_read_argfile (fdtd3d_base_1_interface.hpp:27-113)
 *   jarvis_mpi_init / jarvis_mpi_final     MPI_Init/Finalize when JV_COMPAT_MPI is defined,
 *                                          else one process (rank 0 of 1)
 *   fdtd3d_blend_elastic_model_mpi_module<SimulateType::pure_forward>
 *                                          link / initialize / mpi_sub_forward / reset_for_next_shot
 *                                          (FD/fdtd3d_3_model_mpi_blend/fdtd3d_blend_elastic_model_mpi_bones.hpp:
 *                                          22-31): jv_open, jv_forward_device into seis_record_p's traces
 *   ...<SimulateType::rtm_forward>         link / initialize / reset_for_next_shot /
 *                                          mpi_sub_forward_for_restruct (:33-44): jv_rtm_forward_pass
 *   ...<SimulateType::rtm_backward>        link / initialize / reset_for_next_shot (:46-55)
 *   ...<SimulateType::rtm_reverse>         link / initialize / reset_for_next_shot (:57-64)
 *   the time-reverse loop of mpi_sub_rtm3d the component calls of RTM/rtm3d_1_model_mpi_blend/
 *                                          rtm3d_blend_elastic_model_mpi_meat.hpp:64-113 on sub_phy_p,
 *                                          sub_pml_p, sub_wrc_p and MigImage, each mapped to one
 *                                          jv_rtm_reverse_op kernel (or to nothing, see below)
 *   MigImage                               RTM/rtm3d_0_image_module/rtm3d_image_bones.hpp: initialize,
 *                                          cuda_cal_correlation_from_wave, cuda_laplace_filter,
 *                                          cuda_source_compensation; image_pp .. Ip_fd, Ipp_laplace ..
 *   rtm3d_blend_model_mpi_module::mpi_sub_rtm3d, device_mpi_sub_rtm3d
 *                                          the whole job on the graph path: jv_open +
 *                                          jv_run_project_shard over the job's ranks
 *
 * The time-reverse loop: libjv updates each wavefield with one kernel over
 * its whole grid, so the reference's split of every update into an "edge"
 * part (computed first and sent to the neighbour subdomains) and an
 * "inside" part collapses: cuda_update_and_mpi_exchange_edge_* does
 * nothing and cuda_update_inside_* runs the update.  The source
 * subtraction is fused into the backward stress update and the imaging
 * condition into the backward velocity update (the last write of the
 * source velocities in a step; the receiver velocities are final there),
 * so cuda_subtract_stress_source records the time index and
 * cuda_cal_correlation_from_wave ends the step.  The boundary store stays
 * on the device, so copy_*_host_storage and extract_boundary_wave (run by
 * the forward pass itself) do nothing, and mpi_wait_batch_id has no
 * exchange to wait for.  The results equal jv_run_project's, bit for bit.
 *
 * Differences a driver sees: x/y/z_divide_num must be 1; failures print the
 * library's message and call std::abort(), as the reference does.
 * GPU_NUM_PER_NODE defaults to 8, the GPUs of a B200 node.
 */
#ifndef JV_JARVIS_COMPAT_HPP
#define JV_JARVIS_COMPAT_HPP

#include <cuda_runtime_api.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "jv/jv.h"

#ifdef JV_COMPAT_MPI
#include <mpi.h>
#endif

#ifndef GPU_NUM_PER_NODE
#define GPU_NUM_PER_NODE 8
#endif
#ifndef JV_COMPAT_REC_WIDTH
#define JV_COMPAT_REC_WIDTH 1
#endif

namespace jarvis {
using std::string;
using std::to_string;

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
inline void jv_compat_check(jv_status s, const char *what) {
    if (s != JV_OK) jv_compat_die(what);
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

// ---------------------------------------------------------------- orders
class GeoConst {
   public:
    static const uint32_t phy_fdorder_half = 4;  // 8th-order staggered interior
    static const uint32_t pml_fdorder_half = 2;  // 4th-order CPML
    static const uint32_t rec_width = JV_COMPAT_REC_WIDTH;
};
using geo_const = GeoConst;
static_assert(GeoConst::rec_width >= 1 && GeoConst::rec_width <= GeoConst::phy_fdorder_half,
              "libjv stores 1..4 boundary layers (JV_COMPAT_REC_WIDTH)");

enum class SimulateType { pure_forward, rtm_forward, rtm_backward, rtm_reverse, fwi };
enum class MemType { paged, pinned, device, paged_device, pinned_device };
enum class MemBlock { single, multiple, puppet };
enum class SaveFormat { binary_fld, binary_raw, ascii_xyz, ascii_grd, ascii_txt };

// ---------------------------------------------------------------- Frame
// Grid geometry: x = rows (fastest), y = cols, z = slices; idx = i + j *
// n_rows + k * n_elem_slice.  The members and their order are the
// reference's, so a Frame's bytes are a .fld header (jv_frame).
struct Frame {
    uint64_t n_elem = 0, n_rows = 0, n_elem_slice = 0;
    uint32_t n_cols = 0, n_slices = 0;
    float d_rows = 0, d_cols = 0, d_slices = 0;
    float l_rows = 0, l_cols = 0, l_slices = 0;
    float r_rows = 0, r_cols = 0, r_slices = 0;
    enum class Type { null = 0, vec = 1, mat = 2, cube = 3, line = 10, mesh = 20, grid = 30 };
    Type type = Type::null;

    Frame() {}
    Frame(uint64_t _n_rows, uint32_t _n_cols = 1, uint32_t _n_slices = 1) { set_n(_n_rows, _n_cols, _n_slices); }
    Frame(uint64_t _n_rows, uint32_t _n_cols, uint32_t _n_slices, float _d_rows, float _d_cols, float _d_slices,
          float _l_rows, float _l_cols, float _l_slices) {
        set_ndl(_n_rows, _n_cols, _n_slices, _d_rows, _d_cols, _d_slices, _l_rows, _l_cols, _l_slices);
    }
    void set_n(uint64_t _n_rows, uint32_t _n_cols = 1, uint32_t _n_slices = 1) {
        set_ndl(_n_rows, _n_cols, _n_slices, 0, 0, 0, 0, 0, 0);
        r_rows = r_cols = r_slices = 0;
    }
    void set_nd(uint64_t _n_rows, float _d_rows) { set_ndl(_n_rows, 1, 1, _d_rows, 0, 0, 0, 0, 0); }
    void set_nd(uint64_t _n_rows, uint32_t _n_cols, float _d_rows, float _d_cols) {
        set_ndl(_n_rows, _n_cols, 1, _d_rows, _d_cols, 0, 0, 0, 0);
    }
    void set_nd(uint64_t _n_rows, uint32_t _n_cols, uint32_t _n_slices, float _d_rows, float _d_cols,
                float _d_slices) {
        set_ndl(_n_rows, _n_cols, _n_slices, _d_rows, _d_cols, _d_slices, 0, 0, 0);
    }
    void set_ndl(uint64_t _n_rows, uint32_t _n_cols, uint32_t _n_slices, float _d_rows, float _d_cols,
                 float _d_slices, float _l_rows, float _l_cols, float _l_slices) {
        jv_frame f;
        jv_frame_make(_n_rows, _n_cols, _n_slices, _d_rows, _d_cols, _d_slices, _l_rows, _l_cols, _l_slices, &f);
        from_jv(f);
    }
    void copy(const Frame &_frame) { *this = _frame; }
    // recomputes the derived members from n, d and l
    void re_setndl() { set_ndl(n_rows, n_cols, n_slices, d_rows, d_cols, d_slices, l_rows, l_cols, l_slices); }
    bool is_mat() const { return type == Type::mat; }
    bool is_mesh() const { return type == Type::mesh; }
    bool is_cube() const { return type == Type::cube; }
    bool is_grid() const { return type == Type::grid; }
    Type get_model_type() const { return type; }
    bool operator==(const Frame &o) const {
        return n_rows == o.n_rows && n_cols == o.n_cols && n_slices == o.n_slices && d_rows == o.d_rows &&
               d_cols == o.d_cols && d_slices == o.d_slices && l_rows == o.l_rows && l_cols == o.l_cols &&
               l_slices == o.l_slices && r_rows == o.r_rows && r_cols == o.r_cols && r_slices == o.r_slices;
    }
    // every a-th node of each axis
    Frame sparse(uint32_t a) const {
        return Frame((n_rows - 1) / a + 1, (n_cols - 1) / a + 1, (n_slices - 1) / a + 1, d_rows * a, d_cols * a,
                     d_slices * a, l_rows, l_cols, l_slices);
    }
    // "_nx_ny_nz_lx_ly_lz", the suffix of the reference's raw file names
    string size_info() const {
        return "_" + to_string(n_rows) + "_" + to_string(n_cols) + "_" + to_string(n_slices) + "_" +
               to_string(l_rows) + "_" + to_string(l_cols) + "_" + to_string(l_slices);
    }
    bool is_empty() const { return n_elem == 0; }
    void print_info(const string &s = "") const {
        std::printf("%s\ngrid_x_num:%5llu; interval:%6g; range:[%g, %g]\ngrid_y_num:%5u; interval:%6g; range:[%g, "
                    "%g]\ngrid_z_num:%5u; interval:%6g; range:[%g, %g]\n",
                    s.c_str(), (unsigned long long)n_rows, d_rows, l_rows, r_rows, n_cols, d_cols, l_cols, r_cols,
                    n_slices, d_slices, l_slices, r_slices);
    }
    jv_frame to_jv() const {
        jv_frame f;
        std::memcpy(&f, this, sizeof(f));
        return f;
    }
    void from_jv(const jv_frame &f) { std::memcpy((void *)this, &f, sizeof(f)); }
};
static_assert(sizeof(Frame) == sizeof(jv_frame), "Frame must keep the reference's 72-byte layout");

// ---------------------------------------------------------------- Field
// A field on a Frame: host storage for the paged/pinned kinds, device
// storage for device, both (a mirror) for paged_device / pinned_device.
template <typename elem_type, MemType mem_type = MemType::paged, MemBlock mem_block = MemBlock::single>
class Field : public Frame {
    static_assert(mem_block == MemBlock::single,
                  "MemBlock::multiple / puppet are the halo exchange's contiguous blocks; libjv keeps the whole "
                  "model on one GPU and has no halo exchange");
    static constexpr bool kHost = mem_type != MemType::device;
    static constexpr bool kDevice =
        mem_type == MemType::device || mem_type == MemType::paged_device || mem_type == MemType::pinned_device;
    static constexpr bool kPinned = mem_type == MemType::pinned || mem_type == MemType::pinned_device;

   public:
    Field() {}
    Field(const Field &) = delete;
    Field &operator=(const Field &) = delete;
    ~Field() { clear(); }

    void alloc(const Frame &_frame) {
        clear();
        Frame::copy(_frame);
        const size_t bytes = (size_t)n_elem * sizeof(elem_type);
        if (kHost && n_elem) {
            if (kPinned) jarvis_handle_cuda_error(cudaMallocHost((void **)&host_, bytes));
            else host_ = new elem_type[n_elem];
            std::memset((void *)host_, 0, bytes);
        }
        if (kDevice && n_elem) {
            jarvis_handle_cuda_error(cudaMalloc((void **)&dev_, bytes));
            jarvis_handle_cuda_error(cudaMemset(dev_, 0, bytes));
        }
    }
    void clear() {
        if (host_) {
            if (kPinned) cudaFreeHost(host_);
            else delete[] host_;
        }
        if (dev_) cudaFree(dev_);
        host_ = nullptr;
        dev_ = nullptr;
    }
    // host storage (device storage for MemType::device, which has no other)
    elem_type *ptr() { return kHost ? host_ : dev_; }
    const elem_type *ptr() const { return kHost ? host_ : dev_; }
    elem_type *host_ptr() { return host_; }
    elem_type *device_ptr() { return dev_; }
    const elem_type *device_ptr() const { return dev_; }
    elem_type &operator()(uint64_t i, uint32_t j = 0, uint32_t k = 0) {
        return host_[i + (uint64_t)j * n_rows + (uint64_t)k * n_elem_slice];
    }
    elem_type operator()(uint64_t i, uint32_t j = 0, uint32_t k = 0) const {
        return host_[i + (uint64_t)j * n_rows + (uint64_t)k * n_elem_slice];
    }
    void copy_h2d() { jarvis_handle_cuda_error(cudaMemcpy(dev_, host_, bytes(), cudaMemcpyHostToDevice)); }
    void copy_d2h() { jarvis_handle_cuda_error(cudaMemcpy(host_, dev_, bytes(), cudaMemcpyDeviceToHost)); }
    void copy_h2d(const cudaStream_t &s) {
        jarvis_handle_cuda_error(cudaMemcpyAsync(dev_, host_, bytes(), cudaMemcpyHostToDevice, s));
    }
    void copy_d2h(const cudaStream_t &s) {
        jarvis_handle_cuda_error(cudaMemcpyAsync(host_, dev_, bytes(), cudaMemcpyDeviceToHost, s));
    }
    // one element of the device storage
    void set_value(elem_type v, uint64_t i, uint32_t j = 0, uint32_t k = 0) {
        jarvis_handle_cuda_error(cudaMemcpy(dev_ + index(i, j, k), &v, sizeof(v), cudaMemcpyHostToDevice));
    }
    elem_type get_value(uint64_t i, uint32_t j = 0, uint32_t k = 0) const {
        elem_type v{};
        jarvis_handle_cuda_error(cudaMemcpy(&v, dev_ + index(i, j, k), sizeof(v), cudaMemcpyDeviceToHost));
        return v;
    }
    // host_single_field::read_raw: n_elem values of a raw file on _frame
    void read_raw(const string &_file_path, const Frame &_frame) {
        static_assert(sizeof(elem_type) == sizeof(float), "raw files hold float32");
        alloc(_frame);
        std::vector<float> buf(n_elem);
        jv_compat_check(jv_raw_read(_file_path.c_str(), n_elem, buf.data()), "read_raw");
        put_host(buf.data());
    }
    // host_single_field::load of a .fld file
    void load(const string &_file_path) {
        static_assert(sizeof(elem_type) == sizeof(float), ".fld files hold float32");
        jv_frame f;
        jv_compat_check(jv_fld_read(_file_path.c_str(), &f, nullptr, 0), "load");
        Frame fr;
        fr.from_jv(f);
        alloc(fr);
        std::vector<float> buf(n_elem);
        jv_compat_check(jv_fld_read(_file_path.c_str(), &f, buf.data(), buf.size()), "load");
        put_host(buf.data());
    }
    // host_single_field::save of the host storage
    void save(const string &_file_path, SaveFormat _format) const { save_values(_file_path, _format, host_); }
    // Field<.., device>::cu_save: the device storage, through a host copy
    // (a field without device storage saves its host values)
    void cu_save(const string &_file_path, SaveFormat _format) const {
        if (!kDevice) {
            save(_file_path, _format);
            return;
        }
        std::vector<elem_type> h(n_elem);
        if (n_elem)
            jarvis_handle_cuda_error(cudaMemcpy(h.data(), dev_, bytes(), cudaMemcpyDeviceToHost));
        save_values(_file_path, _format, h.data());
    }

   private:
    elem_type *host_ = nullptr;
    elem_type *dev_ = nullptr;
    size_t bytes() const { return (size_t)n_elem * sizeof(elem_type); }
    uint64_t index(uint64_t i, uint32_t j, uint32_t k) const { return i + (uint64_t)j * n_rows + (uint64_t)k * n_elem_slice; }
    void put_host(const float *src) {
        if (kHost) std::memcpy((void *)host_, src, bytes());
        if (kDevice) jarvis_handle_cuda_error(cudaMemcpy(dev_, src, bytes(), cudaMemcpyHostToDevice));
    }
    // the reference's writers (META/.jarvis_2_field/jarvis_1_host_field_meat.hpp:81-197)
    void save_values(const string &path, SaveFormat fmt, const elem_type *v) const {
        static_assert(sizeof(elem_type) == sizeof(float), "the writers take float32 fields");
        FILE *fp = nullptr;
        switch (fmt) {
        case SaveFormat::binary_fld: {
            const jv_frame f = to_jv();
            jv_compat_check(jv_fld_write(path.c_str(), &f, (const float *)v), "save binary_fld");
            return;
        }
        case SaveFormat::binary_raw:
            fp = std::fopen((path + size_info() + ".raw").c_str(), "wb");
            if (!fp) jv_compat_die("save binary_raw");
            std::fwrite(v, sizeof(elem_type), (size_t)n_elem, fp);
            break;
        case SaveFormat::ascii_xyz:
            if (type != Type::grid) jv_compat_die("save ascii_xyz needs a grid frame");
            fp = std::fopen((path + ".txt").c_str(), "w");
            if (!fp) jv_compat_die("save ascii_xyz");
            for (uint64_t idx = 0; idx < n_elem; ++idx) {
                const double x = l_rows + (double)(idx % n_elem_slice % n_rows) * d_rows;
                const double y = l_cols + (double)(idx % n_elem_slice / n_rows) * d_cols;
                const double z = l_slices + (double)(idx / n_elem_slice) * d_slices;
                std::fprintf(fp, "%7.3f,%7.3f,%7.3f,%8.6e\n", x, y, z, (double)v[idx]);
            }
            break;
        case SaveFormat::ascii_grd: {
            if (type != Type::mesh) jv_compat_die("save ascii_grd needs a mesh frame");
            fp = std::fopen((path + ".grd").c_str(), "w");
            if (!fp) jv_compat_die("save ascii_grd");
            float lo = n_elem ? v[0] : 0.f, hi = lo;
            for (uint64_t q = 0; q < n_elem; q++) {
                lo = v[q] < lo ? v[q] : lo;
                hi = v[q] > hi ? v[q] : hi;
            }
            std::fprintf(fp, "DSAA\n%llu %u\n%g %g\n%g %g\n%g %g\n", (unsigned long long)n_rows, n_cols, l_rows,
                         r_rows, l_cols, r_cols, lo, hi);
            for (uint32_t j = 0; j < n_cols; ++j) {
                for (uint64_t i = 0; i < n_rows; ++i) std::fprintf(fp, "%g ", (double)v[i + j * n_rows]);
                std::fprintf(fp, "\n");
            }
            break;
        }
        case SaveFormat::ascii_txt:
            if (type == Type::null) jv_compat_die("save ascii_txt: frame type is null");
            fp = std::fopen((path + ".txt").c_str(), "wt");
            if (!fp) jv_compat_die("save ascii_txt");
            if (type == Type::cube || type == Type::grid) {
                for (uint32_t k = 0; k < n_slices; ++k)
                    for (uint32_t j = 0; j < n_cols; ++j)
                        for (uint64_t i = 0; i < n_rows; ++i)
                            std::fprintf(fp, "%d,%d,%d,%10.6e\n", (int)i, (int)j, (int)k,
                                         (double)v[i + j * n_rows + k * n_elem_slice]);
            } else {  // one line per column: traces [n_recv][nt] on Frame(nt, n_recv)
                for (uint32_t j = 0; j < n_cols; ++j) {
                    for (uint64_t i = 0; i < n_rows; ++i) std::fprintf(fp, "%10.6e\t", (double)v[i + j * n_rows]);
                    std::fprintf(fp, "\n");
                }
            }
            break;
        }
        std::fclose(fp);
    }
};

// ---------------------------------------------------------------- config
struct ArgList {
    string proj_path, model_path, shot_path, recv_path, output_path;
    int mpi_rank = 0, mpi_size = 1;
    int x_divide_num = 1, y_divide_num = 1, z_divide_num = 1, slots_per_node = 1;
    int pml_num = 0, t_snap = -1;
    float fm = 0.f, T = 0.f, dt = 0.f;
    bool is_output = false;

    void mpi_read_arg_file(string _proj_path, int _mpi_rank, int _mpi_size) {
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

// The reference's per-rank stream/communicator set.  libjv keeps one stream
// per context and has no halo exchange, so there is nothing to wait for.
struct jarvis_global_mpicu_Stream_t {
    int x_divide_num = 1, y_divide_num = 1, z_divide_num = 1, mpi_rank = 0, mpi_size = 1, slots_per_node = 1;
    void initialize(int x, int y, int z, int rank, int size, int slots) {
        x_divide_num = x; y_divide_num = y; z_divide_num = z;
        mpi_rank = rank; mpi_size = size; slots_per_node = slots;
    }
    void mpi_wait_batch_id(int) {}
    void clear() {}
};

// the halo-exchange operator a module's time loop waits on (an id only)
struct jv_compat_halo {
    int operator_id = 0;
};

class elastic_fdtd3d_module_Base {
   public:
    inline static jarvis_global_mpicu_Stream_t *jarvis_mpi_cuda_stream_p = nullptr;
    inline static ArgList *arg_list_p = nullptr;
};

// ---------------------------------------------------------------- the job
namespace jv_compat_detail {
inline jv_ctx *open(const ArgList &a) {
    if (a.x_divide_num * a.y_divide_num * a.z_divide_num != 1)
        std::fprintf(stderr, "[jv] x/y/z_divide_num must be 1: every rank holds the whole model\n");
    jv_options o;
    jv_options_default(&o);
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) o.device = dev;
    o.rec_width = (int)GeoConst::rec_width;
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

struct SeisRecord;

// One job's context and the state of its time-reverse loop, shared by the
// modules linked to one local model.
struct jv_compat_job {
    jv_ctx *ctx = nullptr;
    jv_info info{};
    SeisRecord *observed = nullptr;  // the modelled traces the migration injects
    int shot = -1;                   // shot of the last RTM forward pass
    int it = 0;                      // time index of the current reverse step
    bool begin_pending = false, reverse_open = false;

    jv_compat_job() = default;
    jv_compat_job(const jv_compat_job &) = delete;  // it owns the context
    jv_compat_job &operator=(const jv_compat_job &) = delete;
    ~jv_compat_job() {
        if (ctx) jv_close(ctx);
    }
    void open_reverse();
    void op(int code, int t) {
        open_reverse();
        jv_compat_check(jv_rtm_reverse_op(ctx, code, t), "time-reverse step");
    }
    void end_reverse() {
        if (reverse_open) jv_compat_check(jv_rtm_reverse_end(ctx), "end of the time-reverse loop");
        reverse_open = false;
    }
};

namespace domain {
struct global {};
struct local {};
}  // namespace domain

// elasticGeoModel<domain>: the model grids; the local model carries the job
template <class D>
struct elasticGeoModel {
    Frame gridphy, gridext;
    int margin = 0;
    jv_compat_job job;
    void initialize() {}
    template <class G>
    void initialize(G *) {}
    void clear() {}
    void host_clear() {}
};

// SubGeometry: shot and receiver counts of the job
struct SubGeometry {
    struct Points {
        int n_elem = 0;
    } shot, sub_recv;
    bool is_have_recv = false;
};

// The traces of one shot ([n_recv][nt] on Frame(nt, n_recv), device) and
// every shot's host copy (FD/fdtd3d_0_base_module/fdtd3d_base_4_seisrecord_bones.hpp).
struct SeisRecord : public elastic_fdtd3d_module_Base {
    SubGeometry *sub_geometry_p = nullptr;
    float fm = 0.f, dt = -1.f, T = 0.f;
    int ntime = 0;
    Field<float, MemType::device> vx_seis, vy_seis, vz_seis;
    std::vector<std::vector<float>> vx_host_vec, vy_host_vec, vz_host_vec;

    void initialize(const jv_info &i) {
        ntime = i.nt;
        const Frame f((uint64_t)i.nt, (uint32_t)(i.n_recv > 0 ? i.n_recv : 1), 1);
        vx_seis.alloc(f);
        vy_seis.alloc(f);
        vz_seis.alloc(f);
    }
    void alloc_host_storage(int n_shot) {
        vx_host_vec.assign(n_shot, {});
        vy_host_vec.assign(n_shot, {});
        vz_host_vec.assign(n_shot, {});
    }
    void copy_seis_into_host(int _i_shot) {
        if (!sub_geometry_p || !sub_geometry_p->is_have_recv) return;
        Field<float, MemType::device> *d[3] = {&vx_seis, &vy_seis, &vz_seis};
        std::vector<float> *h[3] = {&vx_host_vec[_i_shot], &vy_host_vec[_i_shot], &vz_host_vec[_i_shot]};
        for (int q = 0; q < 3; q++) {
            h[q]->resize(d[q]->n_elem);
            jarvis_handle_cuda_error(cudaMemcpy(h[q]->data(), d[q]->device_ptr(), d[q]->n_elem * sizeof(float),
                                                cudaMemcpyDeviceToHost));
        }
    }
    void copy_seis_from_host(int _i_shot) {
        if (!sub_geometry_p || !sub_geometry_p->is_have_recv) return;
        Field<float, MemType::device> *d[3] = {&vx_seis, &vy_seis, &vz_seis};
        std::vector<float> *h[3] = {&vx_host_vec[_i_shot], &vy_host_vec[_i_shot], &vz_host_vec[_i_shot]};
        for (int q = 0; q < 3; q++)
            jarvis_handle_cuda_error(cudaMemcpy(d[q]->device_ptr(), h[q]->data(), d[q]->n_elem * sizeof(float),
                                                cudaMemcpyHostToDevice));
    }
};

inline void jv_compat_job::open_reverse() {
    if (!begin_pending) return;
    if (!observed) jv_compat_die("the time-reverse loop needs the modelled traces (link pure_forward first)");
    jv_compat_check(jv_rtm_reverse_begin(ctx, shot, observed->vx_seis.device_ptr(), observed->vy_seis.device_ptr(),
                                         observed->vz_seis.device_ptr()),
                    "start of the time-reverse loop");
    begin_pending = false;
    reverse_open = true;
}

// The wavefield of a module: owned by the library context, so there is
// nothing to zero or free from here (every pass starts from zero).
struct elasticWave {
    void set_zero() {}
    void clear() {}
};

// The physical-domain update of one module; see the header comment for how
// the reference's per-step calls map onto libjv's kernels.
template <SimulateType simulate_type>
struct mpicuPhy {
    jv_compat_job *job = nullptr;
    jv_compat_halo mpi_multi_halo_vel, mpi_multi_halo_stress;
    void set_zero() {}
    void clear() {}
    void cuda_update_and_mpi_exchange_edge_vel() {}
    void cuda_update_and_mpi_exchange_edge_stress() {}
    void cuda_update_inside_vel() {
        static_assert(simulate_type == SimulateType::rtm_backward || simulate_type == SimulateType::rtm_reverse,
                      "modelling passes run as a whole: mpi_sub_forward / mpi_sub_forward_for_restruct");
        job->op(simulate_type == SimulateType::rtm_backward ? JV_OP_BACKWARD_VEL_IMAGE : JV_OP_REVERSE_VEL, job->it);
    }
    void cuda_update_inside_stress() {
        static_assert(simulate_type == SimulateType::rtm_backward || simulate_type == SimulateType::rtm_reverse,
                      "modelling passes run as a whole: mpi_sub_forward / mpi_sub_forward_for_restruct");
        job->op(simulate_type == SimulateType::rtm_backward ? JV_OP_BACKWARD_STRESS : JV_OP_REVERSE_STRESS, job->it);
    }
    // fused into the backward stress update of the same step
    void cuda_subtract_stress_source(int it, int) {
        static_assert(simulate_type == SimulateType::rtm_backward, "the source is subtracted on the backward pass");
        job->it = it;
    }
    void cuda_rtm_reverse_add_vel_source(int it, SeisRecord *seis) {
        static_assert(simulate_type == SimulateType::rtm_reverse, "adjoint sources go into the receiver wavefield");
        job->it = it;
        if (seis && seis != job->observed) {
            if (job->reverse_open) jv_compat_die("the adjoint sources changed inside a time-reverse loop");
            job->observed = seis;
        }
        job->op(JV_OP_INJECT_RECEIVERS, it);
    }
};

// The absorbing layers of a module: only the receiver wavefield's run
// step by step (the modelling passes run as a whole).
struct mpicuCPML {
    jv_compat_job *job = nullptr;
    bool receiver_side = false;
    jv_compat_halo mpi_multi_halo_vel, mpi_multi_halo_stress;
    void set_zero() {}
    void clear() {}
    void cuda_update_and_mpi_exchange_edge_vel() {
        if (!receiver_side) jv_compat_die("modelling passes run as a whole");
        job->op(JV_OP_REVERSE_VEL_PML, job->it);
    }
    void cuda_update_and_mpi_exchange_edge_stress() {
        if (!receiver_side) jv_compat_die("modelling passes run as a whole");
        job->op(JV_OP_REVERSE_STRESS_PML, job->it);
    }
};

// The VOWR boundary store (FD/fdtd3d_0_base_module/fdtd3d_base_5_wave_recon_meat.hpp):
// kept on the device and written by the forward pass itself; the replays
// are kernels of the time-reverse loop.
struct elasticWaveRecon {
    jv_compat_job *job = nullptr;
    void extract_boundary_wave(int) {}
    void copy_into_host_storage(int) {}
    void copy_stress_from_host_storage(int) {}
    void copy_vel_from_host_storage(int) {}
    void inject_boundary_stress(int rec) { job->op(JV_OP_INJECT_BOUNDARY_STRESS, rec); }
    void inject_boundary_vel(int rec) { job->op(JV_OP_INJECT_BOUNDARY_VEL, rec); }
};

template <SimulateType simulate_type>
class fdtd3d_blend_elastic_model_mpi_module;

class fdtd3d_blend_elastic_model_mpi_module_Base : public elastic_fdtd3d_module_Base {
   public:
    elasticGeoModel<domain::global> *glb_model_p = nullptr;
    elasticGeoModel<domain::local> *sub_model_p = nullptr;
    SubGeometry *sub_survey_p = nullptr;
    elasticWave *sub_wave_p = nullptr;
    mpicuCPML *sub_pml_p = nullptr;
    SeisRecord *seis_record_p = nullptr;
};

// Forward modelling of one shot at a time; the traces land in
// seis_record_p->v?_seis (device, Frame(nt, n_recv)).  The module owns the
// objects link() creates, the local model (and with it the job's context)
// among them.
template <>
class fdtd3d_blend_elastic_model_mpi_module<SimulateType::pure_forward>
    : public fdtd3d_blend_elastic_model_mpi_module_Base {
   public:
    mpicuPhy<SimulateType::pure_forward> *sub_phy_p = nullptr;
    int n_recv = 0, nt = 0, n_shot = 0;

    ~fdtd3d_blend_elastic_model_mpi_module() {
        delete sub_phy_p;
        delete seis_record_p;
        delete sub_pml_p;
        delete sub_wave_p;
        delete sub_survey_p;
        delete sub_model_p;
        delete glb_model_p;
    }
    void link() {
        glb_model_p = new elasticGeoModel<domain::global>();
        sub_model_p = new elasticGeoModel<domain::local>();
        sub_wave_p = new elasticWave();
        sub_survey_p = new SubGeometry();
        seis_record_p = new SeisRecord();
        sub_pml_p = new mpicuCPML();
        sub_phy_p = new mpicuPhy<SimulateType::pure_forward>();
        seis_record_p->sub_geometry_p = sub_survey_p;
        sub_model_p->job.observed = seis_record_p;
        sub_pml_p->job = sub_phy_p->job = &sub_model_p->job;
    }
    // the reference's form takes the ArgList from the module base; this one
    // sets it first
    void link(ArgList *_arg_list_p) {
        arg_list_p = _arg_list_p;
        link();
    }
    void initialize() {
        if (!arg_list_p || !sub_model_p) jv_compat_die("initialize before link");
        jv_compat_job &j = sub_model_p->job;
        if (!j.ctx) j.ctx = jv_compat_detail::open(*arg_list_p);
        jv_get_info(j.ctx, &j.info);
        const jv_info &i = j.info;
        n_recv = i.n_recv;
        nt = i.nt;
        n_shot = i.n_shot;
        sub_model_p->gridphy = Frame(i.grid.nx, i.grid.ny, i.grid.nz, i.grid.dx, i.grid.dy, i.grid.dz, 0, 0, 0);
        sub_model_p->margin = i.grid.pml;
        sub_model_p->gridext =
            Frame(i.grid.nx + 2 * i.grid.pml, i.grid.ny + 2 * i.grid.pml, i.grid.nz + 2 * i.grid.pml, i.grid.dx,
                  i.grid.dy, i.grid.dz, -i.grid.pml * i.grid.dx, -i.grid.pml * i.grid.dy, -i.grid.pml * i.grid.dz);
        sub_survey_p->shot.n_elem = n_shot;
        sub_survey_p->sub_recv.n_elem = n_recv;
        sub_survey_p->is_have_recv = n_recv > 0;
        seis_record_p->fm = arg_list_p->fm;
        seis_record_p->dt = arg_list_p->dt;
        seis_record_p->T = arg_list_p->T;
        seis_record_p->initialize(i);
        seis_record_p->alloc_host_storage(n_shot);
    }
    void mpi_sub_forward(int _i_shot) {
        jv_compat_job &j = sub_model_p->job;
        if (!j.ctx) jv_compat_die("mpi_sub_forward before initialize");
        j.end_reverse();
        jv_compat_check(jv_forward_device(j.ctx, _i_shot, seis_record_p->vx_seis.device_ptr(),
                                          seis_record_p->vy_seis.device_ptr(), seis_record_p->vz_seis.device_ptr()),
                        "mpi_sub_forward");
    }
    // every pass starts from a zero wavefield in libjv
    void reset_for_next_shot() {}
};

// The forward pass of RTM with the VOWR boundary store.
template <>
class fdtd3d_blend_elastic_model_mpi_module<SimulateType::rtm_forward>
    : public fdtd3d_blend_elastic_model_mpi_module_Base {
   public:
    mpicuPhy<SimulateType::rtm_forward> *sub_phy_p = nullptr;
    elasticWaveRecon *sub_wrc_p = nullptr;

    ~fdtd3d_blend_elastic_model_mpi_module() {
        delete sub_wrc_p;
        delete sub_phy_p;
        delete sub_pml_p;
        delete seis_record_p;
        delete sub_wave_p;
    }
    void link(elasticGeoModel<domain::local> *_sub_model_p, SubGeometry *_sub_survey_p) {
        sub_model_p = _sub_model_p;
        sub_survey_p = _sub_survey_p;
        sub_wave_p = new elasticWave();
        seis_record_p = new SeisRecord();
        sub_pml_p = new mpicuCPML();
        sub_phy_p = new mpicuPhy<SimulateType::rtm_forward>();
        sub_wrc_p = new elasticWaveRecon();
        sub_pml_p->job = sub_phy_p->job = sub_wrc_p->job = &sub_model_p->job;
    }
    // the receiver wavefield and the store are allocated by the first pass
    void initialize() {}
    void reset_for_next_shot() {}
    void mpi_sub_forward_for_restruct(int _i_shot) {
        jv_compat_job &j = sub_model_p->job;
        if (!j.ctx) jv_compat_die("mpi_sub_forward_for_restruct before the modelling module's initialize");
        j.end_reverse();
        jv_compat_check(jv_rtm_forward_pass(j.ctx, _i_shot), "mpi_sub_forward_for_restruct");
        j.shot = _i_shot;
    }
};
using fdtd3d_for_restruct_M = fdtd3d_blend_elastic_model_mpi_module<SimulateType::rtm_forward>;

// The source wavefield carried back in time (reconstruction).
template <>
class fdtd3d_blend_elastic_model_mpi_module<SimulateType::rtm_backward>
    : public fdtd3d_blend_elastic_model_mpi_module_Base {
   public:
    mpicuPhy<SimulateType::rtm_backward> *sub_phy_p = nullptr;
    elasticWaveRecon *sub_wrc_p = nullptr;

    ~fdtd3d_blend_elastic_model_mpi_module() { delete sub_phy_p; }
    void link(fdtd3d_for_restruct_M *_fdtd3d_for_for_restruct_p) {
        sub_model_p = _fdtd3d_for_for_restruct_p->sub_model_p;
        sub_wave_p = _fdtd3d_for_for_restruct_p->sub_wave_p;
        sub_survey_p = _fdtd3d_for_for_restruct_p->sub_survey_p;
        sub_wrc_p = _fdtd3d_for_for_restruct_p->sub_wrc_p;
        seis_record_p = _fdtd3d_for_for_restruct_p->seis_record_p;
        sub_phy_p = new mpicuPhy<SimulateType::rtm_backward>();
        sub_phy_p->job = &sub_model_p->job;
    }
    void initialize() {}
    // the loop starts (cleared receiver wavefield and shot image) at its
    // first kernel
    void reset_for_next_shot() { sub_model_p->job.begin_pending = true; }
};

// The receiver wavefield propagated backward from the recorded traces.
template <>
class fdtd3d_blend_elastic_model_mpi_module<SimulateType::rtm_reverse>
    : public fdtd3d_blend_elastic_model_mpi_module_Base {
   public:
    mpicuPhy<SimulateType::rtm_reverse> *sub_phy_p = nullptr;

    ~fdtd3d_blend_elastic_model_mpi_module() {
        delete sub_phy_p;
        delete sub_pml_p;
        delete seis_record_p;
        delete sub_wave_p;
    }
    void link(elasticGeoModel<domain::local> *_sub_model_p, SubGeometry *_sub_survey_p) {
        sub_model_p = _sub_model_p;
        sub_survey_p = _sub_survey_p;
        sub_wave_p = new elasticWave();
        seis_record_p = new SeisRecord();
        sub_pml_p = new mpicuCPML();
        sub_pml_p->receiver_side = true;
        sub_phy_p = new mpicuPhy<SimulateType::rtm_reverse>();
        sub_pml_p->job = sub_phy_p->job = &sub_model_p->job;
    }
    void initialize() {}
    void reset_for_next_shot() { sub_model_p->job.begin_pending = true; }
};

// The image stacks (RTM/rtm3d_0_image_module/rtm3d_image_bones.hpp): the
// correlation runs inside the backward velocity update; at the end of the
// job cuda_laplace_filter / cuda_source_compensation fill the fields below
// (device, gridphy) from jv_image_finalize.
struct MigImage {
    jarvis_global_mpicu_Stream_t *jarvis_mpi_cuda_stream_p = nullptr;
    fdtd3d_blend_elastic_model_mpi_module<SimulateType::rtm_backward> *fdtd_restruct_p = nullptr;
    fdtd3d_blend_elastic_model_mpi_module<SimulateType::rtm_reverse> *fdtd_reverse_p = nullptr;
    Field<float, MemType::device> image_pp, image_ps, image_sp, image_ss, Ip_fd;
    Field<float, MemType::device> Ipp_laplace, Ips_laplace, Isp_laplace, Iss_laplace;

    void link(jarvis_global_mpicu_Stream_t *_stream_p,
              fdtd3d_blend_elastic_model_mpi_module<SimulateType::rtm_backward> *_fdtd_restruct_p,
              fdtd3d_blend_elastic_model_mpi_module<SimulateType::rtm_reverse> *_fdtd_reverse_p) {
        jarvis_mpi_cuda_stream_p = _stream_p;
        fdtd_restruct_p = _fdtd_restruct_p;
        fdtd_reverse_p = _fdtd_reverse_p;
    }
    void initialize() {
        jv_compat_job &j = job();
        const Frame &g = fdtd_restruct_p->sub_model_p->gridphy;
        Field<float, MemType::device> *all[9] = {&image_pp, &image_ps, &image_sp, &image_ss, &Ip_fd,
                                                 &Ipp_laplace, &Ips_laplace, &Isp_laplace, &Iss_laplace};
        for (auto *f : all) f->alloc(g);
        jv_compat_check(jv_image_reset(j.ctx), "MigImage::initialize");
        finalized_ = false;
    }
    // the zero-lag correlation of this step ran in the backward velocity
    // update; after the last step (it == 0) the shot joins the stacks
    void cuda_cal_correlation_from_wave() {
        jv_compat_job &j = job();
        if (j.reverse_open && j.it == 0) j.end_reverse();
    }
    void cuda_laplace_filter() { finalize(); }
    void cuda_source_compensation() { finalize(); }

   private:
    bool finalized_ = false;
    jv_compat_job &job() { return fdtd_restruct_p->sub_model_p->job; }
    // Laplacian of the uncompensated stacks, then the compensation
    // (RTM/rtm3d_1_model_mpi_blend/rtm3d_blend_elastic_model_mpi_meat.hpp:123-124)
    void finalize() {
        if (finalized_) return;
        jv_compat_job &j = job();
        j.end_reverse();
        const size_t n = image_pp.n_elem;
        std::vector<float> h(8 * n);
        float *o[8];
        for (int q = 0; q < 8; q++) o[q] = h.data() + q * n;
        jv_compat_check(jv_image_finalize(j.ctx, o[0], o[1], o[2], o[3], o[4], o[5], o[6], o[7]), "image finalize");
        Field<float, MemType::device> *dst[8] = {&image_pp, &image_ps, &image_sp, &image_ss,
                                                 &Ipp_laplace, &Ips_laplace, &Isp_laplace, &Iss_laplace};
        for (int q = 0; q < 8; q++)
            jarvis_handle_cuda_error(cudaMemcpy(dst[q]->device_ptr(), o[q], n * sizeof(float), cudaMemcpyHostToDevice));
        std::vector<double> ip(n);
        jv_compat_check(jv_image_get(j.ctx, JV_IMG_IP, ip.data()), "Ip_fd");
        std::vector<float> ipf(ip.begin(), ip.end());
        jarvis_handle_cuda_error(cudaMemcpy(Ip_fd.device_ptr(), ipf.data(), n * sizeof(float), cudaMemcpyHostToDevice));
        finalized_ = true;
    }
};

// The RTM job: its four modules and the image, linked as the reference
// links them.  mpi_sub_rtm3d runs the whole job on the graph path
// (jv_run_project_shard, the job's ranks each taking their share of the
// shots); a driver may instead run the modules' own loops in the shape of
// the reference's mpi_sub_rtm3d, with the same results.
class rtm3d_blend_model_mpi_module : public elastic_fdtd3d_module_Base {
   public:
    fdtd3d_blend_elastic_model_mpi_module<SimulateType::pure_forward> fdtd_seisdata;
    fdtd3d_blend_elastic_model_mpi_module<SimulateType::rtm_forward> fdtd_rtm_forward;
    fdtd3d_blend_elastic_model_mpi_module<SimulateType::rtm_backward> fdtd_rtm_backward;
    fdtd3d_blend_elastic_model_mpi_module<SimulateType::rtm_reverse> fdtd_rtm_reverse;
    MigImage image;

    void link(ArgList *_arg_list_p, jarvis_global_mpicu_Stream_t *_stream_p) {
        arg_list_p = _arg_list_p;
        jarvis_mpi_cuda_stream_p = _stream_p;
        fdtd_seisdata.link();
        fdtd_rtm_forward.link(fdtd_seisdata.sub_model_p, fdtd_seisdata.sub_survey_p);
        fdtd_rtm_backward.link(&fdtd_rtm_forward);
        fdtd_rtm_reverse.link(fdtd_seisdata.sub_model_p, fdtd_seisdata.sub_survey_p);
        image.link(jarvis_mpi_cuda_stream_p, &fdtd_rtm_backward, &fdtd_rtm_reverse);
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

}  // namespace jarvis

#endif /* JV_JARVIS_COMPAT_HPP */
