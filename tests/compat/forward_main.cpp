// Forward modelling through the jarvis pure_forward module names over
// libjv: writes shot 0's vz traces as raw float32 to argv[2].
#include "jv/jarvis_compat.hpp"
using namespace jarvis;

int main(int argc, char *argv[]) {
    jarvis_mpi_init(argc, argv, mpi_rank, mpi_size);
    if (argc < 3) return 2;
    jarvis_handle_cuda_error(cudaSetDevice(mpi_rank % GPU_NUM_PER_NODE));
    ArgList arg_list;
    arg_list.mpi_read_arg_file(argv[1], mpi_rank, mpi_size);
    fdtd3d_blend_elastic_model_mpi_module<SimulateType::pure_forward> fwd;
    fwd.link(&arg_list);
    fwd.initialize();
    fwd.reset_for_next_shot();
    fwd.mpi_sub_forward(0);
    fwd.seis_record_p->copy_seis_into_host(0);
    const std::vector<float> &vz = fwd.seis_record_p->vz_host_vec[0];
    FILE *f = std::fopen(argv[2], "wb");
    if (!f) return 3;
    std::fwrite(vz.data(), sizeof(float), vz.size(), f);
    std::fclose(f);
    std::printf("n_recv %d nt %d n_shot %d\n", fwd.n_recv, fwd.nt, fwd.n_shot);
    jarvis_mpi_final;
    return 0;
}
