// jv_internal.hpp -- device data layout and kernel interfaces of libjv.
//
// Layout in HBM
//   Every wavefield component and model parameter covers gridext
//   (gridphy + pml cells per face) in one pitched array:
//       elem(i, j, k) = base + xoff + i + sy * j + sz * k
//   with the row pitch sy a multiple of 32 floats and xoff chosen so that
//   the first gridphy column (i = pml) starts on a 128-byte boundary.
//   Absorbing-layer memory variables live only in the six boundary slabs
//   (slab-local dense indexing), not on the full grid.
#pragma once

#include <cstddef>
#include <cstdint>

namespace jv {

constexpr int kPhyHalf = 4;  // GeoConst::phy_fdorder_half (8th-order interior)
constexpr int kPmlHalf = 2;  // GeoConst::pml_fdorder_half (4th-order CPML)

// SimulateType of FD/fdtd3d_0_base_module/fdtd3d_base_1_interface.hpp:19-26
enum Mode : int { kFwd = 0, kRtmFwd = 1, kBwd = 2, kRev = 3 };

// wavefield components
enum Fld : int { VX = 0, VY, VZ, SXX, SYY, SZZ, SXY, SXZ, SYZ, SAU, VXP, VYP, VZP, kNumFld };

struct GridDev {
    int nx, ny, nz;   // gridext
    int m;            // margin (pml_num)
    int px, py, pz;   // gridphy
    long long sy, sz; // pitches in elements
    long long xoff;   // offset of gridext (0,0,0) from the array base
    float dx, dy, dz; // spacing
};

struct WaveDev {
    float *f[kNumFld];
};

// One CPML slab: cells [x0,x1) x [y0,y1) x [z0,z1) of gridext, processed
// in 4-cell x groups starting at the 16-byte aligned cell gstart (cells of
// a group outside [x0,x1) are masked).  Its memory variables are 6*naxes
// arrays of `stride` floats: rows of `pitch` = 4*ngroups floats, group g
// of row (y,z) at psi_off + ((z-z0)*(y1-y0) + (y-y0))*pitch + 4g; array
// q = 3*axis + t for the velocity update, 3*naxes + 3*axis + t for the
// stress update (axis 0 = x, 1 = y, 2 = z).  Launch shape: blocks of
// 256 threads, thread t -> group t % gx, row t / gx (gx * gy <= 256),
// bx*by blocks per plane.
struct PmlSlab {
    int x0, x1, y0, y1, z0, z1;
    int gstart, ngroups;
    int gx, gy, bx, by;
    int first_block;
    int naxes, pitch;
    long long psi_off, stride;
};

struct CpmlDev {
    PmlSlab s[6];
    int nslab, nblocks;
    int zp;                   // planes a thread updates (1 or 2); blocks cover zp planes
    float dt;                 // |time step|
    const float4 *ax[3];      // per axis, per extended index: {K, K_half, alpha, alpha_half}, K = 0 outside
    float *psi;               // this wavefield's memory-variable arena
};

// The image of the shot being migrated: FP32 accumulators over its time
// steps, as the reference keeps them (RTM/rtm3d_0_image_module/
// rtm3d_iamge_kernel.hpp:6-51, RTM = src/jarvis_cpp/jarvis/.jarvis_2_app/
// .jarvis_3_seismology/elastic_1_rtm3d_model_mpi); added into the FP64
// stacks at the end of the shot.
struct ImageDev {
    float *ip, *pp, *ps, *sp, *ss;  // gridphy, dense x-fastest
};

// The stacks over shots (FP64), gridphy, dense x-fastest.
struct StackDev {
    double *ip, *pp, *ps, *sp, *ss;
};

struct SegDev {          // one VOWR face box
    int fld;
    int x0, nxb, y0, nyb, z0, nzb;
    long long off;       // offset in the packed per-step record
    long long nblk_first;
    int vw;              // values a thread moves: 4 (16-byte accesses along x rows) or 1
};

// The VOWR boundary store and its face boxes.  Boxes of the velocity
// fields come first; each box is cut into blocks of 256 threads of vw
// cells each, and a block's box is the last one whose first block is not
// after it.
// boundary-store precision (the values of jv_precision)
constexpr int kStoreF32 = 0, kStoreBF16 = 1, kStoreFP16 = 2;

constexpr int kVowrMaxSegs = 64;  // face boxes of a record: at most 10 fields x 6 faces

struct VowrDev {
    // the face boxes, in block order, passed to the kernels in their
    // (constant-bank) parameters: a block finds its box without a load from
    // global memory
    SegDev seg[kVowrMaxSegs];
    int vel_blocks, all_blocks;
    long long per_step;  // values of one step's record
    int nslot;           // records in the store
    float *store;        // FP32 records (prec == JV_FP32)
    // 16-bit records (prec == JV_BF16 / JV_FP16): value / scale, one FP32
    // scale per face box and step (scales[slot * nseg + box]) = the box's
    // largest magnitude; amax[2][nseg] collects it, by step parity
    int prec;
    int nseg;
    uint16_t *store16;
    float *scales;
    unsigned *amax;
};

// Per-step state in device memory, read by the kernels of a captured
// time loop, so one CUDA graph serves every shot and every step.
struct StepState {
    int it;              // current time step
    int pad;
    long long src;       // element index of the shot's source node
    float *tr[3];        // recorded traces (vx, vy, vz), [nrec][nt]
    const float *obs[3]; // traces injected into the receiver wavefield
};

// TMA descriptor of one field array (a CUtensorMap, opaque outside
// kernels.cu): the pitched gridext array as a 3-D tensor, boxes of one
// plane of a row tile with its x/y halo.
struct alignas(64) FieldMap {
    unsigned char bytes[128];
};
// Descriptors for the z-marching stress kernel (variant 3) of one
// wavefield: planes of vx, vy, vz with their x/y halo, and core tiles (the
// tile's cells only) of vx, vy, vz, lam, mu and the seven stress fields;
// and its launch facts.
constexpr int kZmCore = 12;  // vx vy vz lam mu sxx syy szz sxy sxz syz sau
struct WaveMaps {
    FieldMap halo[3];
    FieldMap core[kZmCore];
    bool ok = false; // false: variant 3 is not available for this grid
    int rows = 0;    // rows of a tile
    int boxw = 0, boxh = 0;  // halo box
    int corew = 0;           // core box width (rows = `rows`)
    int ntx = 1, tpp = 0;    // x tiles and the x pairs of each (even when ntx > 1)
    int nsm = 0;     // CTAs of the persistent grid
    int *err = nullptr;  // device flag: a bounded wait in the kernel ran out
};

// Geometry of the full-gridext stress kernel (variant 4).
//  - x tiles: tile xt holds the physical x pairs [xt TPP, (xt+1) TPP) of the
//    hxi = px/2, the first also the low absorbing strip [2, m), the last the
//    high one [m+px, nx-2) (one tile: both); hxe: absorbing pairs a tile
//    row carries (m-2 with one tile, else (m-2)/2); tpad: 4 TPP rounded up
//    to whole warps (4 TPP where the rounding alone would take the tile
//    past one CTA), the first thread of the absorbing pairs; corew: the
//    core box width (the widest tile's).  ytiles, nzi: 4-row tiles over y in
//    [2, ny-2), planes z in [2, nz-2).
//  - The stress memory variables of this kernel are axis-major: per axis
//    three arrays over the cells that absorb on that axis, rows packed
//    (x arrays [t][z-2][y-2][xc], pitch PX over xc = the W absorbing x
//    columns; y arrays [t][z-2][yc][x-2] and z arrays [t][zc][y-2][x-2],
//    pitch PY over x-2), so that a tile's memory variables arrive by TMA
//    with its fields (y and z boxes PB wide, from the tile's first cell
//    rounded down to 16 bytes).  W = 2 (m - 2) absorbing indices per axis.
//  - Runs: each tile's planes are cut into Q chunks of L planes (the last
//    one padded with idle items); run r = chunk * (NTX ytiles) + tile, tile
//    = yt NTX + xt, and CTA b takes runs b, b + grid, ...  Neighbouring CTAs
//    then march neighbouring tiles through the same planes together, so
//    halo rows are shared in L2.
struct FzGeo {
    int corew;
    int hxi, hxe, tpad;
    int NTX, TPP;       // x tiles; physical x pairs per tile
    int ytiles, nzi;
    int PX, PY, PB, W;  // PB: width of a y/z memory-variable box
    int Q, L, R;
    float *psx, *psy, *psz;
    const float4 *ax[3];
};

// floats of one set (3 axes x 3 arrays) of axis-major memory variables; a
// wavefield holds two, the velocity set first, then the stress set
long long fz_psi_floats(const GridDev &g);

// TMA descriptors of the full-gridext stress kernel of one wavefield
struct FullMaps {
    FieldMap halo[3];             // vx vy vz
    FieldMap core[kZmCore + 1];   // vx vy vz, lam, mu, vp, sxx syy szz sxy sxz syz, sau
    FieldMap psi[3];              // the x, y and z memory-variable arrays (4-D: 3 arrays each)
    // the velocity kernel's: halo planes sxy syy syz, bands sxx sxz, core
    // tiles rho vp vx vy vz, window feed sxz syz szz, memory variables
    FieldMap vhalo[3], vband[2], vcore[5], vfeed[3], vpsi[3];
    bool ok = false;              // false: variant 4 is not available for this grid
    FzGeo geo{}, vgeo{};          // stress and velocity kernels (their memory-variable sets differ)
    int threads = 0;
    int grid = 0;
    size_t smem = 0, vsmem = 0;
    int *err = nullptr;
    int qcand[3] = {0, 0, 0};     // the cost model's three best run-chunk counts, best first
};

// interior-kernel choice: variant 0 = one z plane per block, 1 = z-marching
// over chunks of zchunk planes (0: the whole column)
struct KCfg {
    int variant = 3;
    int zchunk = 0;
    int gx = 0, gy = 0;  // variant 2 block: x groups per block, rows per block (0: auto)
    int minb = 4;        // variant 2: blocks per SM the register budget is set for (3 or 4)
    int pml_minb = 4;    // CPML kernels: the same
    int zp = 1;          // variant 2: z planes per thread (1 or 2)
    int pml_zp = 1;      // CPML kernels: the same
    int fzq = 0;         // variant 4: run chunks per tile (0: the cost model's choice)
};

// kernels.cu ------------------------------------------------------------
// vp, dt / rho (the velocity update's density term), lambda, mu on gridext
int k_model_prep(const GridDev &g, const float *d_vp_phy, const float *d_vs_phy, const float *d_rho_phy, float dt,
                 float *vp, float *bdt, float *lam, float *mu, void *stream);
int k_zero_range(float *p, size_t n, void *stream);

int k_vel_phy(int mode, const GridDev &g, const WaveDev &w, const float *bdt, float dt, int rec_w,
              const WaveDev *rev, const ImageDev *img, const KCfg &kc, void *stream);

// it_off: the kernels of a step read the time step as st->it + it_off (a
// captured chunk of steps advances st->it once, at its end)
int k_stress_phy(int mode, const GridDev &g, const WaveDev &w, const float *lam, const float *mu, float dt,
                 int rec_w, const float *wavelet, const StepState *st, int it_off, const KCfg &kc, void *stream,
                 const WaveMaps *maps = nullptr);
// Builds the TMA descriptors of w's velocity fields for variant 3's
// z-marching stress kernel (also variant 4's source reconstruction).  Rows
// of more than 248 cells are cut into x tiles of an even number of pairs.
// maps->ok stays false when those tiles would have fewer than 384 threads,
// or the driver entry point is missing.  Returns a cudaError_t.
int k_make_wave_maps(const GridDev &g, const WaveDev &w, const float *lam, const float *mu, int *err_flag,
                     WaveMaps *maps);
// The descriptors of the full-gridext stress kernel (variant 4), with the
// run schedule cut into `chunks` chunks per tile (0: the cost model's
// choice; maps->qcand lists its three best); maps->ok
// stays false when the grid does not suit it (odd pml_num or nx, a tile
// row of more than 512 threads or a halo row wider than 256 floats, the
// driver entry point missing).  Returns a cudaError_t.
int k_make_full_maps(const GridDev &g, const WaveDev &w, const float *lam, const float *mu, const float *vp,
                     const float *bdt, float4 *const ax[3], float *psi, int *err_flag, int chunks,
                     FullMaps *maps);
// Stress update of every updated cell of gridext, interior and absorbing
// layers in one launch (modes kFwd, kRtmFwd, kRev).
int k_stress_full(int mode, const GridDev &g, const WaveDev &w, float dt, const float *wavelet, const StepState *st,
                  int it_off, const FullMaps &maps, void *stream);
// Velocity update of every updated cell of gridext (variant 4; vx, vy, vz)
int k_vel_full(const GridDev &g, const WaveDev &w, float dt, const FullMaps &maps, void *stream);
int k_vel_pml(const GridDev &g, const CpmlDev &c, const WaveDev &w, const float *bdt, const float *vp,
              const KCfg &kc, void *stream);
int k_stress_pml(const GridDev &g, const CpmlDev &c, const WaveDev &w, const float *lam, const float *mu,
                 const float *vp, int with_sau, const KCfg &kc, void *stream);

int k_record(const WaveDev &w, const long long *rec, int nrec, int nt, const StepState *st, int it_off,
             void *stream);
int k_inject_rec(const WaveDev &w, const long long *rec, int nrec, int nt, const StepState *st, int it_off,
                 void *stream);
// pack (1) or unpack (0) record st->it + slot_shift; which: 0 all fields,
// 1 the velocity fields, 2 the stress fields
// Packs (pack = 1) or unpacks the face boxes of step st->it + slot_shift;
// which = 0 all boxes, 1 velocity boxes, 2 stress boxes.  With a 16-bit
// store, packing is two launches: the boxes' largest magnitudes, then the
// scaled values.
int k_vowr(const GridDev &g, const WaveDev &w, const VowrDev &v, const StepState *st, int slot_shift, int pack,
           int which, void *stream);
int k_step_advance(StepState *st, int delta, void *stream);
int k_image_finalize(const GridDev &g, const StackDev &img, float *out /* 8 arrays */, void *stream);
// stack += shot image (FP64 sums of the FP32 shot accumulators)
int k_image_stack(const GridDev &g, const ImageDev &shot, const StackDev &stack, void *stream);
// FP64 energy of the velocity and stress fields of w over gridphy, added into *out
int k_wave_energy(const GridDev &g, const WaveDev &w, double *out, void *stream);
int upload_coefficients(const float list[5][4], const float dc2[2]);
int k_count_nonfinite(const void *p, size_t n, int is_double, unsigned long long *out, void *stream);

}  // namespace jv
