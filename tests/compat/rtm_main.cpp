// A driver written against the jarvis class names (the shape of the
// reference's RTM main: MPI init, device choice, ArgList, stream set,
// module link, device_mpi_sub_rtm3d), built against libjv through
// jv/jarvis_compat.hpp.  Usage: rtm_main <project dir with trailing />
#include "jv/jarvis_compat.hpp"
using namespace jarvis;

int main(int argc, char *argv[]) {
    jarvis_mpi_init(argc, argv, mpi_rank, mpi_size);
    if (argc < 2) {
        std::printf("usage: %s <project path>\n", argv[0]);
        return 2;
    }
    MPI_Barrier(MPI_COMM_WORLD);
    std::string proj_path = std::string(argv[1]);
    jarvis_handle_cuda_error(cudaSetDevice(mpi_rank % GPU_NUM_PER_NODE));
    jarvis_get_gpu_memory(mpi_rank % GPU_NUM_PER_NODE);
    jarvis_global_mpicu_Stream_t jarvis_mpi_cuda_stream;
    ArgList arg_list;
    rtm3d_blend_model_mpi_module rtm_mpi;
    arg_list.mpi_read_arg_file(proj_path, mpi_rank, mpi_size);
    jarvis_mpi_cuda_stream.initialize(arg_list.x_divide_num, arg_list.y_divide_num, arg_list.z_divide_num, mpi_rank,
                                      mpi_size, arg_list.slots_per_node);
    rtm_mpi.link(&arg_list, &jarvis_mpi_cuda_stream);
    device_mpi_sub_rtm3d(&rtm_mpi);
    jarvis_mpi_final;
    return 0;
}
