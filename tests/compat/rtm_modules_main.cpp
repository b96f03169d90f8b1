// A driver that runs the RTM job through the four module specialisations
// and the image, in the shape of the reference's mpi_sub_rtm3d
// (RTM/rtm3d_1_model_mpi_blend/rtm3d_blend_elastic_model_mpi_meat.hpp:18-135):
// model every shot and save its traces, then per shot the forward pass for
// the reconstruction and the time-reverse loop of component calls, then
// the Laplacian, the compensation and the saved images.  Built against
// libjv through jv/jarvis_compat.hpp.  Usage: rtm_modules_main <project dir/>
#include "jv/jarvis_compat.hpp"
using namespace jarvis;

int main(int argc, char *argv[]) {
    jarvis_mpi_init(argc, argv, mpi_rank, mpi_size);
    if (argc < 2) return 2;
    jarvis_handle_cuda_error(cudaSetDevice(mpi_rank % GPU_NUM_PER_NODE));
    jarvis_global_mpicu_Stream_t stream;
    ArgList arg_list;
    arg_list.mpi_read_arg_file(argv[1], mpi_rank, mpi_size);
    stream.initialize(arg_list.x_divide_num, arg_list.y_divide_num, arg_list.z_divide_num, mpi_rank, mpi_size,
                      arg_list.slots_per_node);
    rtm3d_blend_model_mpi_module rtm;
    rtm.link(&arg_list, &stream);
    auto &fdtd_seisdata = rtm.fdtd_seisdata;
    auto &fdtd_rtm_forward = rtm.fdtd_rtm_forward;
    auto &fdtd_rtm_backward = rtm.fdtd_rtm_backward;
    auto &fdtd_rtm_reverse = rtm.fdtd_rtm_reverse;
    auto &image = rtm.image;
    jarvis_global_mpicu_Stream_t *jarvis_mpi_cuda_stream_p = &stream;

    fdtd_seisdata.initialize();
    for (int ishot = 0; ishot < fdtd_seisdata.sub_survey_p->shot.n_elem; ishot++) {
        fdtd_seisdata.reset_for_next_shot();
        fdtd_seisdata.mpi_sub_forward(ishot);
        fdtd_seisdata.seis_record_p->copy_seis_into_host(ishot);
        if (fdtd_seisdata.sub_survey_p->is_have_recv) {
            const string pre = arg_list.output_path + "v";
            const string suf = "_seis_" + to_string(arg_list.mpi_rank) + "_" + to_string(ishot);
            fdtd_seisdata.seis_record_p->vx_seis.cu_save(pre + "x" + suf, SaveFormat::ascii_txt);
            fdtd_seisdata.seis_record_p->vy_seis.cu_save(pre + "y" + suf, SaveFormat::ascii_txt);
            fdtd_seisdata.seis_record_p->vz_seis.cu_save(pre + "z" + suf, SaveFormat::ascii_txt);
        }
        MPI_Barrier(MPI_COMM_WORLD);
    }
    fdtd_seisdata.sub_wave_p->clear();
    fdtd_seisdata.sub_pml_p->clear();
    fdtd_seisdata.sub_phy_p->clear();
    jarvis_mpi_cuda_stream_p->clear();

    fdtd_rtm_forward.initialize();
    fdtd_rtm_backward.initialize();
    fdtd_rtm_reverse.initialize();
    image.initialize();
    for (int ishot = 0; ishot < fdtd_seisdata.sub_survey_p->shot.n_elem; ishot++) {
        fdtd_seisdata.seis_record_p->copy_seis_from_host(ishot);
        fdtd_rtm_forward.reset_for_next_shot();
        fdtd_rtm_forward.mpi_sub_forward_for_restruct(ishot);
        fdtd_rtm_backward.reset_for_next_shot();
        fdtd_rtm_reverse.reset_for_next_shot();
        for (int it = fdtd_seisdata.seis_record_p->ntime - 1; it >= 0; it--) {
            // UPDATE 1
            fdtd_rtm_backward.sub_phy_p->cuda_subtract_stress_source(it, ishot);
            fdtd_rtm_reverse.sub_phy_p->cuda_rtm_reverse_add_vel_source(it, fdtd_seisdata.seis_record_p);
            fdtd_rtm_backward.sub_phy_p->cuda_update_and_mpi_exchange_edge_stress();
            fdtd_rtm_reverse.sub_phy_p->cuda_update_and_mpi_exchange_edge_vel();
            fdtd_rtm_reverse.sub_pml_p->cuda_update_and_mpi_exchange_edge_vel();
            fdtd_rtm_backward.sub_phy_p->cuda_update_inside_stress();
            fdtd_rtm_backward.sub_wrc_p->inject_boundary_stress(it - 1);
            fdtd_rtm_backward.sub_wrc_p->copy_stress_from_host_storage(it - 2);
            fdtd_rtm_reverse.sub_phy_p->cuda_update_inside_vel();
            jarvis_mpi_cuda_stream_p->mpi_wait_batch_id(fdtd_rtm_reverse.sub_pml_p->mpi_multi_halo_vel.operator_id);
            jarvis_mpi_cuda_stream_p->mpi_wait_batch_id(fdtd_rtm_reverse.sub_phy_p->mpi_multi_halo_vel.operator_id);
            jarvis_mpi_cuda_stream_p->mpi_wait_batch_id(fdtd_rtm_backward.sub_phy_p->mpi_multi_halo_stress.operator_id);
            // UPDATE 2
            fdtd_rtm_backward.sub_phy_p->cuda_update_and_mpi_exchange_edge_vel();
            fdtd_rtm_reverse.sub_phy_p->cuda_update_and_mpi_exchange_edge_stress();
            fdtd_rtm_reverse.sub_pml_p->cuda_update_and_mpi_exchange_edge_stress();
            fdtd_rtm_backward.sub_phy_p->cuda_update_inside_vel();
            fdtd_rtm_backward.sub_wrc_p->inject_boundary_vel(it - 1);
            fdtd_rtm_backward.sub_wrc_p->copy_vel_from_host_storage(it - 2);
            fdtd_rtm_reverse.sub_phy_p->cuda_update_inside_stress();
            image.cuda_cal_correlation_from_wave();
            jarvis_mpi_cuda_stream_p->mpi_wait_batch_id(fdtd_rtm_reverse.sub_pml_p->mpi_multi_halo_stress.operator_id);
            jarvis_mpi_cuda_stream_p->mpi_wait_batch_id(fdtd_rtm_reverse.sub_phy_p->mpi_multi_halo_stress.operator_id);
            jarvis_mpi_cuda_stream_p->mpi_wait_batch_id(fdtd_rtm_backward.sub_phy_p->mpi_multi_halo_vel.operator_id);
        }
    }
    image.cuda_laplace_filter();
    image.cuda_source_compensation();
    const string rank = to_string(arg_list.mpi_rank);
    image.image_pp.cu_save(arg_list.output_path + "image_pp_" + rank, SaveFormat::binary_raw);
    image.Ipp_laplace.cu_save(arg_list.output_path + "image_pp_laplace_" + rank, SaveFormat::binary_raw);
    image.image_ps.cu_save(arg_list.output_path + "image_ps_" + rank, SaveFormat::binary_raw);
    image.image_sp.cu_save(arg_list.output_path + "image_sp_" + rank, SaveFormat::binary_raw);
    image.image_ss.cu_save(arg_list.output_path + "image_ss_" + rank, SaveFormat::binary_raw);
    image.Ip_fd.cu_save(arg_list.output_path + "image_ipfd_" + rank, SaveFormat::binary_raw);
    image.image_pp.cu_save(arg_list.output_path + "image_pp_" + rank, SaveFormat::binary_fld);
    std::printf("geo_const: %u %u %u\n", geo_const::phy_fdorder_half, geo_const::pml_fdorder_half,
                geo_const::rec_width);
    jarvis_mpi_final;
    return 0;
}
