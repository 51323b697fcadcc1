// Timing harness over the reference build (CPU baseline; test
// infrastructure only).
//
//   sdpa_ref_iter DATA.dat-s PARAM.sdpa WARMUP STEPS [KAPPA]
//
// Sets the problem up exactly as pinpal (sdpa_main.cpp:43-292), runs WARMUP
// untimed passes of its main loop, then STEPS timed passes of the stock loop
// body (sdpa_main.cpp:294-376, no captured copies), and prints one JSON
// object: per-pass wall seconds and the reference's own ComputeTime deltas
// per pass for the Schur build ("Make bMat", sdpa_newton.cpp:1223-1244) and
// the Cholesky of B ("Cholesky bMat", sdpa_newton.cpp:1246-1299).
#include <sdpa_io.h>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <omp.h>

extern "C" {
void *ref_open(const char *dataFile, const char *paramFile, double kappa);
int ref_step(void *h);
int ref_dims(void *h, int *out, int cap);
void ref_set_capture(void *h, int on);
void ref_times(void *h, double *out);
}

int main(int argc, char **argv) {
    if (argc < 5) {
        std::fprintf(stderr, "usage: %s DATA PARAM WARMUP STEPS [KAPPA]\n", argv[0]);
        return 2;
    }
    double kappa = argc > 5 ? std::atof(argv[5]) : 1.2;
    int warm = std::atoi(argv[3]), steps = std::atoi(argv[4]);
    auto t0 = std::chrono::steady_clock::now();
    void *h = ref_open(argv[1], argv[2], kappa);
    if (!h) {
        std::fprintf(stderr, "cannot open %s\n", argv[1]);
        return 1;
    }
    double tsetup = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    ref_set_capture(h, 0);
    int dims[64];
    ref_dims(h, dims, 64);
    for (int i = 0; i < warm; ++i)
        if (ref_step(h) != 0) {
            std::fprintf(stderr, "solver stopped during warm-up\n");
            return 1;
        }
    std::vector<double> wall, schur, chol;
    for (int i = 0; i < steps; ++i) {
        double t0[2], t1[2];
        ref_times(h, t0);
        auto a = std::chrono::steady_clock::now();
        int rc = ref_step(h);
        double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - a).count();
        if (rc != 0) {
            std::fprintf(stderr, "solver stopped at timed pass %d (rc=%d)\n", i, rc);
            return 1;
        }
        ref_times(h, t1);
        wall.push_back(dt);
        schur.push_back(t1[0] - t0[0]);
        chol.push_back(t1[1] - t0[1]);
    }
    auto list = [](const char *key, const std::vector<double> &v) {
        std::printf(", \"%s\": [", key);
        for (size_t i = 0; i < v.size(); ++i) std::printf("%s%.6f", i ? ", " : "", v[i]);
        std::printf("]");
    };
    std::printf("{\"m\": %d, \"nblock\": %d, \"threads\": %d, \"setup_s\": %.6f", dims[0], dims[1], omp_get_max_threads(), tsetup);
    list("pass_s", wall);
    list("schur_s", schur);
    list("chol_s", chol);
    std::printf("}\n");
    return 0;
}
