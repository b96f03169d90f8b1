// project_io.hpp -- the reference's project files, read and written in C++.
//
//  argfile.json  JSON with // comments, ArgList keys
//                (FD/fdtd3d_0_base_module/fdtd3d_base_1_interface.hpp:27-113)
//  shot/rece     count, then "x y z" per point
//                (src/jarvis_cpp/jarvis/.jarvis_1_util/.jarvis_2_geometry/jarvis_device_geometry_meat.hpp:6-54)
//  .gms model    240-byte header, per parameter a 64-byte name + data, z fastest, then x, then y
//                (src/jarvis_cpp/jarvis/.jarvis_1_util/.jarvis_0_gms/jarvis_device_gms_meat.hpp:11-79)
//  traces        "%10.6e\t" per sample, one line per receiver
//                (.jarvis_0_meta/.jarvis_2_field/jarvis_1_host_field_meat.hpp:159-197)
//  images        raw float32 with Frame::size_info() in the name
//                (.jarvis_0_meta/.jarvis_2_field/jarvis_0_frame_meat.hpp:347-351)
//  raw models    one float32 file per parameter, x fastest, with its Frame given
//                by the caller (host_single_field::read_raw,
//                .jarvis_0_meta/.jarvis_2_field/jarvis_1_host_field_meat.hpp:65-79)
//  .fld fields   the Frame struct's bytes, then the data
//                (save_as_binary_fld / load, jarvis_1_host_field_meat.hpp:41-64,81-89)
// (FD = src/jarvis_cpp/jarvis/.jarvis_2_app/.jarvis_3_seismology/elastic_1_fdtd3d_model_mpi)
#pragma once

#include <map>
#include <string>
#include <vector>

namespace jv {

struct ArgFile {
    std::string proj_path, model_path, shot_path, recv_path, output_path;
    int x_divide_num = 1, y_divide_num = 1, z_divide_num = 1, slots_per_node = 1;
    int pml_num = 0, t_snap = -1;
    float fm = 0.f, T = 0.f, dt = 0.f;
    bool is_output = false;
    int rec_width = 0;       // optional key (0: not given)
    std::string precision;   // optional key
    // optional raw model: vp/vs/rho files (prefixed with proj_path) on the
    // Frame n_rows x n_cols x n_slices, d_rows/d_cols/d_slices; when vp_path
    // is given, model_path is not read
    std::string vp_path, vs_path, rho_path;
    int n_rows = 0, n_cols = 0, n_slices = 0;
    float d_rows = 0.f, d_cols = 0.f, d_slices = 0.f;
    bool save_fld = false;   // optional key: also write the images as .fld
};

// Parses proj_path + "argfile.json".  Returns "" on success, else a message.
std::string read_argfile(const std::string &proj_path, ArgFile *a);
std::string read_points(const std::string &path, std::vector<float> *xyz);

struct GmsModel {
    int nx = 0, ny = 0, nz = 0;
    float dx = 0, dy = 0, dz = 0, lx = 0, ly = 0, lz = 0;
    std::vector<std::vector<float>> params;  // each nx*ny*nz, x fastest
};
std::string read_gms(const std::string &path, GmsModel *m);

// a raw model (vp, vs, rho files of nx*ny*nz floats, x fastest)
std::string read_raw_model(const ArgFile &a, GmsModel *m);
// exactly n floats from a raw file
std::string read_raw(const std::string &path, float *out, size_t n);

std::string size_info(int nx, int ny, int nz, float lx, float ly, float lz);
std::string write_traces(const std::string &path_noext, const float *tr, int nrec, int nt);
std::string write_raw(const std::string &path, const float *a, size_t n);

}  // namespace jv
