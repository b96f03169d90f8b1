// Frame and Field of the jarvis front end on host memory (no GPU needed):
// builds a grid Frame, reads a raw float32 file onto it (Field::read_raw),
// saves it as .fld and .raw, loads the .fld back (Field::load) and prints
// what it found.  Usage: field_main <dir/> (with dir/in.raw of 4*3*2 floats)
#include "jv/jarvis_compat.hpp"
using namespace jarvis;

int main(int argc, char *argv[]) {
    if (argc < 2) return 2;
    const string d = argv[1];
    static_assert(geo_const::phy_fdorder_half == 4 && geo_const::pml_fdorder_half == 2, "orders");
    Frame g(4, 3, 2, 10.f, 10.f, 5.f, -20.f, 0.f, 2.5f);
    Field<float, MemType::paged> a;
    a.read_raw(d + "in.raw", g);
    a(1, 2, 1) += 100.f;
    a.save(d + "out", SaveFormat::binary_fld);
    a.save(d + "out", SaveFormat::binary_raw);
    a.save(d + "out_xyz", SaveFormat::ascii_xyz);
    Field<float, MemType::paged> b;
    b.load(d + "out.fld");
    const bool same_frame = b == a && b.type == Frame::Type::grid && b.size_info() == a.size_info();
    float diff = 0.f;
    for (uint64_t q = 0; q < a.n_elem; q++) diff += std::abs(a.ptr()[q] - b.ptr()[q]);
    Frame s = g.sparse(2);
    std::printf("frame %d type %d r %g %g %g diff %g sparse %llu %u %u %g\n", same_frame ? 1 : 0, (int)b.type,
                b.r_rows, b.r_cols, b.r_slices, diff, (unsigned long long)s.n_rows, s.n_cols, s.n_slices, s.d_rows);
    std::printf("%s\n", a.size_info().c_str());
    return 0;
}
