// suite3d_impl.hpp -- host-side state of one 3D chunk, shared by the
// kernel-interface layer (suite3d.cu) and the device-resident driver
// (driver3d.cu). Same design as the 2D suite (suite2d_impl.hpp).
#pragma once

#include "kernels3d.cuh"

#include <cuda_runtime.h>

enum AltField3 { ALT3_P = 0, ALT3_U = 1, ALT3_R = 2, ALT3_SD = 3, ALT3_COUNT = 4 };

struct TlSuite3D {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    tl3d::Geo g{0, 0, 0, 0};
    void* slab = nullptr;
    size_t slab_bytes = 0;
    tl::ReduceSlots rs{};
    double* h_out = nullptr;
    long partial_capacity = 0;
    State* d_states = nullptr;
    int d_states_cap = 0;
    double* d_comm = nullptr;
    long d_comm_cap = 0;
    double* alt[ALT3_COUNT] = {nullptr, nullptr, nullptr, nullptr};
    tl::Profiler prof;
    struct {
        bool calc_p = false;
        double beta = 0.0;
        int halo[TL3_NUM_FIELDS] = {0, 0, 0, 0, 0, 0};
    } pend;
    tl::DevState* d_state = nullptr;
    int* h_mirror = nullptr;
    int* d_mirror = nullptr;
    double* d_cg_alphas = nullptr;
    double* d_cg_betas = nullptr;
    double* d_cheby_alphas = nullptr;
    double* d_cheby_betas = nullptr;
    int table_len = 0;
};

#define TL3_LAUNCH(s, name, ...)               \
    do {                                       \
        (s)->prof.begin((s)->stream, name);    \
        __VA_ARGS__;                           \
        (s)->prof.end((s)->stream);            \
        TL_LAUNCHED(name);                     \
    } while (0)

namespace tl3d {

TlSuite3D* suite_of(Chunk* chunk);
inline dim3 interior_grid(const Geo& g)
{
    return dim3(tl::ceil_div(g.x - 2 * g.hd, BX), tl::ceil_div(g.y - 2 * g.hd, BY), tl::ceil_div(g.z - 2 * g.hd, g.zr));
}
// z cells per thread of the interior sweeps: the grid should be whole waves
// both for the staged stencil sweeps (TL3D_MINB blocks per SM) and for the
// pointwise ones (8 per SM); longer pencils carry less prologue (one extra
// staged plane per pencil).
inline int choose_zr(int nx, int ny, int nz, int sm_count)
{
    const long bxy = (long)tl::ceil_div(nx, BX) * tl::ceil_div(ny, BY);
    int best = ZR;
    double best_score = -1.0;
    for (int zr = 4; zr <= 32; ++zr) {
        const long blocks = bxy * tl::ceil_div(nz, zr);
        auto eff = [&](long slots) {
            const long waves = (blocks + slots - 1) / slots;
            return (double)blocks / (double)(waves * slots);
        };
        const double score = eff((long)sm_count * TL3D_MINB) * eff((long)sm_count * 8) * zr / (zr + 1.0);
        if (score > best_score + 1e-12) {
            best_score = score;
            best = zr;
        }
    }
    return best;
}
inline dim3 full_grid(const Geo& g) { return dim3(tl::ceil_div(g.x, FBX), tl::ceil_div(g.y, FBY), g.z); }
// Interior grid plus the halo-duty z-plane of the fused sweeps.
inline dim3 fused_grid(const Geo& g)
{
    dim3 d = interior_grid(g);
    d.z += 1;
    return d;
}
inline dim3 interior_block() { return dim3(BX, BY); }
inline dim3 full_block() { return dim3(FBX, FBY); }
bool fetch(TlSuite3D* s, int n, double* out);
void flush(TlSuite3D* s, Chunk* chunk);
Faces faces_of(const Chunk* chunk);
double** field_slot(Chunk* chunk, AltField3 f);
void swap_alt(TlSuite3D* s, Chunk* chunk, AltField3 f);

}  // namespace tl3d
