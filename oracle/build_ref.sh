#!/usr/bin/env bash
# Builds the reference's own RTM driver (RTM/rtm3d_2_model_mpi_blend_test:
# rtm3d_blend_elastic_model_mpi_main.cpp + _device.cu) as a CHECKER for the
# oracle.  Test infrastructure only: nothing in the product links it.
#
# The reference sources are copied to a scratch directory OUTSIDE the
# repository, patched there, and compiled; only the binaries land in
# oracle/_ref/ (git-ignored).  No reference source enters the repository.
#
# Patches (each a minimal change; the numerical kernels are untouched):
#  1. FD/fdtd3d_0_base_module/fdtd3d_base_3_geomodel_meat.hpp:415-438 --
#     the reference ignores model_path and loads a hard-coded salt model
#     from the author's home directory; re-enable its own commented-out
#     GmsReader lines and drop the salt block, so model_path (a .gms file
#     with vp, vs, rho) is read.
#  2. same file, :480 -- drop cuda_smooth_model(): its result is never
#     read (the host copies of lambda/mu/rho feed the local model) and
#     smooth_model_y_dir reads one row past the end of the array at the
#     last y row of the last slice.
#  3. FD/fdtd3d_0_base_module/fdtd3d_base_1_interface.hpp:15 --
#     GeoConst::rec_width becomes the compile-time value JVREF_REC_WIDTH.
#  4. FD/fdtd3d_0_base_module/fdtd3d_base_4_seisrecord_meat.hpp:64,353 and
#     FD/fdtd3d_2_phy_mpi_module/fdtd3d_phy_mpi_4_device_meat.hpp:319 --
#     the receiver kernels launch <<<1, n_recv>>>, which fails above 1024
#     receivers; launch ceil(n/128) blocks of 128 and index by the global
#     thread id instead.
#  5. RTM/rtm3d_1_model_mpi_blend/rtm3d_blend_elastic_model_mpi_meat.hpp:131
#     -- also save Ip_fd and the ps/sp/ss images (the reference saves only
#     image_pp and its Laplacian).
#
# Usage: [JV_REFERENCE_ROOT=<reference checkout>] oracle/build_ref.sh [rec_width ...]   (default: 1 4)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
# the reference checkout: JV_REFERENCE_ROOT, else a sibling of this repository
REF=${JV_REFERENCE_ROOT:-$(cd "$HERE/../.." && pwd)/reference}
OUT="$HERE/_ref"
WIDTHS=("$@")
if [ ${#WIDTHS[@]} -eq 0 ]; then WIDTHS=(1 4); fi
if [ ! -d "$REF/src/jarvis_cpp" ]; then
    echo "build_ref.sh: reference tree not found at $REF" >&2
    exit 3
fi
SCR=$(mktemp -d /tmp/jvref_build.XXXXXX)
trap 'rm -rf "$SCR"' EXIT
mkdir -p "$OUT" "$SCR/.external"
cp -r "$REF/src" "$SCR/src"
cp -r "$REF/.external/json" "$SCR/.external/json"
ln -s /usr/local/cuda/include "$SCR/.external/cuda"
chmod -R u+w "$SCR"

J="$SCR/src/jarvis_cpp/jarvis/.jarvis_2_app/.jarvis_3_seismology"
FD="$J/elastic_1_fdtd3d_model_mpi"
RTM="$J/elastic_1_rtm3d_model_mpi"
GEO="$FD/fdtd3d_0_base_module/fdtd3d_base_3_geomodel_meat.hpp"

# 1. model_path -> GmsReader (vp, vs, rho), no hard-coded salt block
sed -i -e 's|^\(\s*\)//GmsReader gms(model_path);|\1GmsReader gms(model_path);|' \
       -e 's|^\(\s*\)//gms.read_gms_by_order_to_ffield(\(phy_[a-z]*\));|\1gms.read_gms_by_order_to_ffield(\2);|' \
       -e 's|^\(\s*\)//gms.clear();|\1gms.clear();|' "$GEO"
sed -i -e '/phy_vp.alloc(Frame(676/,/gridphy = phy_vp;/{/gridphy = phy_vp;/!d}' "$GEO"
# 2. no device smoothing (unused result, out-of-bounds read)
sed -i -e 's|^\(\s*\)cuda_smooth_model(20, 4, 1);|\1/* smoothing removed by build_ref.sh */|' "$GEO"
grep -q "GmsReader gms(model_path);" "$GEO"
! grep -q "salt_model" "$GEO"
! grep -q "^\s*cuda_smooth_model(" "$GEO"
# 3. rec_width from the command line
IF="$FD/fdtd3d_0_base_module/fdtd3d_base_1_interface.hpp"
sed -i -e 's|static const uint32_t rec_width = 1;|static const uint32_t rec_width = JVREF_REC_WIDTH;|' "$IF"
grep -q "rec_width = JVREF_REC_WIDTH" "$IF"
# 4. receiver kernels above 1024 receivers
SR="$FD/fdtd3d_0_base_module/fdtd3d_base_4_seisrecord_meat.hpp"
PH="$FD/fdtd3d_2_phy_mpi_module/fdtd3d_phy_mpi_4_device_meat.hpp"
sed -i -e '64s|int iRece = threadIdx.x;|int iRece = threadIdx.x + blockDim.x * blockIdx.x;|' "$SR"
sed -i -e 's|(void \*)sub_cal_seis_data_base, 1, sub_geometry_p->sub_recv.n_elem,|(void *)sub_cal_seis_data_base, (sub_geometry_p->sub_recv.n_elem + 127) / 128, 128,|' "$SR"
sed -i -e 's|(void \*)sub_rtm_reverse_add_vel_source, 1, sub_geometry_p->sub_recv.n_elem,|(void *)sub_rtm_reverse_add_vel_source, (sub_geometry_p->sub_recv.n_elem + 127) / 128, 128,|' "$PH"
sed -n 64p "$SR" | grep -q "blockIdx.x"
grep -q "sub_cal_seis_data_base, (sub_geometry_p" "$SR"
grep -q "sub_rtm_reverse_add_vel_source, (sub_geometry_p" "$PH"
# 5. save every image
RB="$RTM/rtm3d_1_model_mpi_blend/rtm3d_blend_elastic_model_mpi_meat.hpp"
sed -i -e '/image.Ipp_laplace.cu_save(/a\
                image.Ip_fd.cu_save(arg_list_p->output_path + "image_ipfd_" + to_string(arg_list_p->mpi_rank), SaveFormat::binary_raw);\
                image.image_ps.cu_save(arg_list_p->output_path + "image_ps_" + to_string(arg_list_p->mpi_rank), SaveFormat::binary_raw);\
                image.image_sp.cu_save(arg_list_p->output_path + "image_sp_" + to_string(arg_list_p->mpi_rank), SaveFormat::binary_raw);\
                image.image_ss.cu_save(arg_list_p->output_path + "image_ss_" + to_string(arg_list_p->mpi_rank), SaveFormat::binary_raw);' "$RB"
grep -q "image_ipfd_" "$RB"

T="$RTM/rtm3d_2_model_mpi_blend_test"
for W in "${WIDTHS[@]}"; do
    B="$SCR/obj_w$W"
    mkdir -p "$B"
    nvcc -std=c++17 -O3 -w -gencode arch=compute_100a,code=sm_100a -DJVREF_REC_WIDTH="$W" \
        -I"$HERE/ref_stub" -c "$T/rtm3d_blend_elastic_model_mpi_device.cu" -o "$B/device.o"
    g++ -std=c++17 -O3 -w -DJVREF_REC_WIDTH="$W" -I"$HERE/ref_stub" -I/usr/local/cuda/include \
        -c "$T/rtm3d_blend_elastic_model_mpi_main.cpp" -o "$B/main.o"
    g++ -o "$OUT/jvref_rtm_w$W" "$B/main.o" "$B/device.o" -L/usr/local/cuda/lib64 -lcudart
    echo "built $OUT/jvref_rtm_w$W"
done
