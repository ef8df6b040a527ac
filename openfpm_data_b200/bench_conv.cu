// Throughput of the conv2_b route against the fixed-function Gray-Scott kernel on one grid.
//
// Usage: bench_conv <map file> <steps> <warmup>
// The map file holds a block map as written by bench.py: int64 n, then keys[n] (int64), then u, v
// ((n + 1) * 512 float32 each, the background chunk last) and mask ((n + 1) * 512 bytes).  The grid
// gets u, v, u', v' (backgrounds 1, 0, 1, 0).  Both routes first run one step from the same state and
// their results are compared bit for bit at the active points; then each runs `steps` steps (after
// `warmup` untimed ones), timed with CUDA events.  Prints one JSON object.
//
// The conv2_b lambda is the Gray-Scott update as a user writes it for the reference's conv2_b
// (src/SparseGridGpu/SparseGridGpu.hpp:2627-2645), in the association order of the library's GS7
// definition.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "openfpm_b200/SparseGridGpu.hpp"

using namespace openfpm_b200;

typedef SparseGridGpu<3, aggregate<float, float, float, float>, 8> Grid4;

int main(int argc, char** argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s <map file> <steps> <warmup>\n", argv[0]);
        return 2;
    }
    const int steps = std::atoi(argv[2]), warmup = std::atoi(argv[3]);
    FILE* fp = std::fopen(argv[1], "rb");
    if (!fp) return 2;
    int64_t n = 0;
    if (std::fread(&n, 8, 1, fp) != 1 || n <= 0) return 2;
    std::vector<int64_t> keys(n);
    std::vector<float> u((n + 1) * 512), v((n + 1) * 512);
    std::vector<uint8_t> mask((n + 1) * 512);
    if (std::fread(keys.data(), 8, n, fp) != (size_t)n || std::fread(u.data(), 4, u.size(), fp) != u.size() ||
        std::fread(v.data(), 4, v.size(), fp) != v.size() || std::fread(mask.data(), 1, mask.size(), fp) != mask.size())
        return 2;
    std::fclose(fp);
    const size_t sz[3] = {512, 512, 512};
    Grid4 grid(sz);
    grid.setBackgroundValue<0>(1.0f);
    grid.setBackgroundValue<1>(0.0f);
    grid.setBackgroundValue<2>(1.0f);
    grid.setBackgroundValue<3>(0.0f);
    const void* data[4] = {u.data(), v.data(), u.data(), v.data()};
    check(sgb_load_map(grid.handle(), n, keys.data(), data, mask.data(), nullptr), "load_map");
    int64_t active = 0;
    for (int64_t i = 0; i < n * 512; ++i) active += (mask[i] & 3) == 1;

    const float Du = 0.16f, Dv = 0.08f, F = 0.035f, K = 0.065f, dt = 1.0f;
    auto gs = [=] __device__(float& uo, float& vo, cp_block<float, 8>& uu, cp_block<float, 8>& vv,
                             data_block<8>& blk, int offset, int i, int j, int k) {
        auto lap = [](cp_block<float, 8>& f, int i, int j, int k) {
            float l = __fmul_rn(-6.0f, f(i, j, k));
            l = __fadd_rn(l, __fadd_rn(f(i - 1, j, k), f(i + 1, j, k)));
            l = __fadd_rn(l, __fadd_rn(f(i, j - 1, k), f(i, j + 1, k)));
            return __fadd_rn(l, __fadd_rn(f(i, j, k - 1), f(i, j, k + 1)));
        };
        (void)blk;
        (void)offset;
        const float uc = uu(i, j, k), vc = vv(i, j, k);
        const float uvv = __fmul_rn(__fmul_rn(uc, vc), vc);
        float du = __fmaf_rn(Du, lap(uu, i, j, k), -uvv);
        du = __fmaf_rn(F, __fsub_rn(1.0f, uc), du);
        float dv = __fmaf_rn(Dv, lap(vv, i, j, k), uvv);
        dv = __fmaf_rn(-(F + K), vc, dv);
        uo = __fmaf_rn(dt, du, uc);
        vo = __fmaf_rn(dt, dv, vc);
    };
    const grid_key_dx<3> lo({0, 0, 0}), hi({511, 511, 511});
    int src[2] = {0, 1}, dst[2] = {2, 3};
    const float prm[5] = {Du, Dv, F, K, dt};

    // one step each from the same state: bit for bit at the active points
    auto download = [&](std::vector<std::vector<float>>& f) {
        std::vector<int64_t> k(n);
        std::vector<uint8_t> m((n + 1) * 512);
        f.assign(4, std::vector<float>((n + 1) * 512));
        void* ptrs[4] = {f[0].data(), f[1].data(), f[2].data(), f[3].data()};
        check(sgb_download_map(grid.handle(), k.data(), ptrs, m.data(), nullptr), "download");
    };
    std::vector<std::vector<float>> G, C;
    check(sgb_apply_stencil(grid.handle(), SGB_GS7, src, dst, prm, 5, nullptr, nullptr), "gs7");
    download(G);
    grid.conv2_b<0, 1, 2, 3, 1>(lo, hi, gs);
    download(C);
    bool equal = true;
    for (int64_t i = 0; i < n * 512 && equal; ++i)
        if ((mask[i] & 3) == 1)
            equal = std::memcmp(&G[2][i], &C[2][i], 4) == 0 && std::memcmp(&G[3][i], &C[3][i], 4) == 0;

    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto time_steps = [&](bool conv) {
        for (int k = 0; k < warmup + steps; ++k) {
            if (k == warmup) cudaEventRecord(e0);
            const bool fwd = k % 2 == 0;
            if (conv) {
                if (fwd) grid.conv2_b<0, 1, 2, 3, 1>(lo, hi, gs);
                else grid.conv2_b<2, 3, 0, 1, 1>(lo, hi, gs);
            } else {
                check(sgb_apply_stencil(grid.handle(), SGB_GS7, fwd ? src : dst, fwd ? dst : src, prm, 5, nullptr,
                                        nullptr),
                      "gs7");
            }
        }
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        return ms / 1e3;
    };
    const double t_gs7 = time_steps(false), t_conv = time_steps(true);
    const double pts = (double)active * steps;
    std::printf("{\"active_points\": %lld, \"steps\": %d, \"gs7_gpts\": %.3f, \"conv2_b_gpts\": %.3f, "
                "\"conv2_b_over_gs7\": %.4f, \"one_step_bit_equal\": %s}\n",
                (long long)active, steps, pts / t_gs7 / 1e9, pts / t_conv / 1e9, t_gs7 / t_conv,
                equal ? "true" : "false");
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
