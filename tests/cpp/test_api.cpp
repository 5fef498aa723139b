// Mirrors cases of the reference's test/core/solver/test_lsqr.cpp and
// test/core/workspace/test_workspace.cpp through the reference-signature
// C++ API (include/tomos/b200.hpp) on the device.  Built and run by
// tests/test_gpu_cpp_api.py; exits non-zero on the first failed check.
#include <cmath>
#include <cstdio>
#include <stdexcept>
#include <vector>

#include "tomos/b200.hpp"

using namespace tomos;

static int failures = 0;
#define CHECK(cond, ...)                              \
    do {                                              \
        if (!(cond)) {                                \
            std::printf("FAIL %s:%d: ", __FILE__, __LINE__); \
            std::printf(__VA_ARGS__);                 \
            std::printf("\n");                        \
            ++failures;                               \
        }                                             \
    } while (0)

static Dense upload(Context& ctx, const std::vector<float>& col_major, std::size_t m, std::size_t n) {
    Dense d = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {m, n});
    cudaMemcpy(d.data(), col_major.data(), sizeof(float) * m * n, cudaMemcpyHostToDevice);
    return d;
}

static std::vector<float> download(Dense& d, std::size_t len) {
    std::vector<float> h(len);
    cudaMemcpy(h.data(), d.data(), sizeof(float) * len, cudaMemcpyDeviceToHost);
    return h;
}

int main() {
    Context ctx(Device::CUDA);

    // 6x3 consistent system, x_true = (1, -1, 2)  (test_lsqr.cpp:203-247).
    {
        const float rows[6][3] = {{4, 1, 0}, {0, 3, 1}, {1, 0, 5}, {2, 1, 1}, {0, 2, 3}, {1, 1, 2}};
        const float xt[3] = {1, -1, 2};
        std::vector<float> a(18), b(6, 0.f);
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 3; ++j) {
                a[i + 6 * j] = rows[i][j];
                b[i] += rows[i][j] * xt[j];
            }
        Dense A = upload(ctx, a, 6, 3), B = upload(ctx, b, 6, 1);
        Dense X = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {3, 1});
        Workspace ws = create_lsqr_workspace(ctx, {6, 3}, NumericType::FP32);
        int iters = 0;
        std::vector<double> hist;
        lsqr_solve(ctx, A, B, X, ws, 1e-7, 200, 1e-7, &iters, &hist);
        auto x = download(X, 3);
        for (int j = 0; j < 3; ++j) CHECK(std::fabs(x[j] - xt[j]) < 2e-5, "x[%d]=%g", j, x[j]);
        CHECK(iters > 0 && (int)hist.size() == iters, "iters=%d hist=%zu", iters, hist.size());
    }

    // Inconsistent 4x2 system: x = (3.5, 1.4).
    {
        std::vector<float> a = {1, 1, 1, 1, 1, 2, 3, 4}, b = {6, 5, 7, 10};
        Dense A = upload(ctx, a, 4, 2), B = upload(ctx, b, 4, 1);
        Dense X = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {2, 1});
        Workspace ws = create_lsqr_workspace(ctx, {4, 2}, NumericType::FP32);
        lsqr_solve(ctx, A, B, X, ws, 1e-10, 200, 1e-10);
        auto x = download(X, 2);
        CHECK(std::fabs(x[0] - 3.5f) < 1e-5 && std::fabs(x[1] - 1.4f) < 1e-5, "x=(%g,%g)", x[0], x[1]);
    }

    // Packed FP32_16 A through split_fp32_16, implicit duplicate, sketch-QR
    // preconditioner (test_lsqr.cpp:461-528 pipeline at 40 x 5).
    {
        const std::size_t m = 4000, n = 40, k = 160;
        std::vector<float> a(m * n), b(m, 0.f), xt(n);
        unsigned s = 12345u;
        auto rnd = [&]() { s = s * 1664525u + 1013904223u; return (float)((s >> 8) & 0xFFFF) / 32768.f - 1.f; };
        for (std::size_t j = 0; j < n; ++j) xt[j] = rnd();
        for (std::size_t j = 0; j < n; ++j)
            for (std::size_t i = 0; i < m; ++i) a[i + m * j] = rnd() * std::pow(10.f, (float)j / n * 2.f);
        for (std::size_t j = 0; j < n; ++j)
            for (std::size_t i = 0; i < m; ++i) b[i] += a[i + m * j] * xt[j];
        Dense A = upload(ctx, a, m, n), B = upload(ctx, b, m, 1);
        Dense P = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32_16, {m, n});
        split_fp32_16(A, P);
        Dense SA = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP64, {k, n});
        apply_count_sketch_hashed(A, SA);
        generate_sketch_qr_precond(SA);
        Dense Rinv = Dense::wrap_strided(ctx, Layout::COL_MAJOR, NumericType::FP64, {n, n}, k, SA.data());
        Workspace ws = create_lsqr_workspace(ctx, {m, n}, NumericType::FP32, NumericType::FP64);
        add_precond(Rinv, ws);
        ws.use_implicit_duplicate_ = true;
        Dense X = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {n, 1});
        int iters = 0;
        lsqr_solve(ctx, P, B, X, ws, 1e-6, 50, 1e-6, &iters, nullptr, 6);
        auto x = download(X, n);
        double err = 0, nrm = 0;
        for (std::size_t j = 0; j < n; ++j) {
            err += (x[j] - xt[j]) * (x[j] - xt[j]);
            nrm += xt[j] * xt[j];
        }
        CHECK(std::sqrt(err / nrm) < 1e-4, "packed rel err %g after %d iterations", std::sqrt(err / nrm), iters);
    }

    // add_precond type mismatch throws std::invalid_argument
    // (test_workspace.cpp:17-79); FP16 storage has no kernel registered.
    {
        Workspace ws = create_lsqr_workspace(ctx, {10, 3}, NumericType::FP32, NumericType::FP64);
        Dense R = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {3, 3});
        bool threw = false;
        try {
            add_precond(R, ws);
        } catch (const std::invalid_argument&) {
            threw = true;
        }
        CHECK(threw, "add_precond type mismatch did not throw");
        threw = false;
        try {
            Dense H = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32_16, {4, 4});
            Dense xv = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {4, 1});
            Dense yv = Dense::create_strided(ctx, Layout::COL_MAJOR, NumericType::FP32, {4, 1});
            mv_apply(Device::CUDA, NO_TRANSPOSE, 1.0, H, xv, 0.0, yv, NumericType::FP64);
        } catch (const std::runtime_error&) {
            threw = true;
        }
        CHECK(threw, "unregistered compute type did not throw");
    }

    if (failures) {
        std::printf("%d failure(s)\n", failures);
        return 1;
    }
    std::printf("cpp api ok\n");
    return 0;
}
