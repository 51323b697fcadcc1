// The reference's command line (sdpa_main.cpp:455-672) and pinpal's file
// handling (sdpa_main.cpp:43-453) over the device solver.
#include "../../include/sddd.h"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>

#include "capi_internal.h"
#include "context.h"
#include "solver.h"

namespace {

void usage(const char *argv0) {
    std::printf("\n*** Please assign data file and output file.***\n\n");
    std::printf("---- option type 1 ------------\n");
    std::printf("%s DataFile OutputFile [InitialPtFile] [-pt parameters]\n", argv0);
    std::printf("parameters = 0 default, 1 fast (unstable), 2 slow (stable)\n");
    std::printf("example1-1: %s example1.dat example1.result\n", argv0);
    std::printf("example1-2: %s example1.dat-s example1.result\n", argv0);
    std::printf("example1-3: %s example1.dat example1.result example1.ini\n", argv0);
    std::printf("example1-4: %s example1.dat example1.result -pt 2\n\n", argv0);
    std::printf("---- option type 2 ------------\n");
    std::printf("%s [option filename]+ \n", argv0);
    std::printf("  -dd : data dense :: -ds : data sparse     \n");
    std::printf("  -id : init dense :: -is : init sparse     \n");
    std::printf("  -o  : output     :: -p  : parameter       \n");
    std::printf("  -pt : parameters , 0 default, 1 fast (unstable)\n");
    std::printf("                     2 slow (stable)         \n");
    std::printf("  -tc : slices (8-16) of the tensor-core split Cholesky of the Schur matrix\n");
    std::printf("  -wd : write the final point, dense  (an init file with 34 digits)\n");
    std::printf("  -ws : write the final point, sparse (an init file with 34 digits)\n");
    std::printf("example2-1: %s -o example1.result -dd example1.dat\n", argv0);
    std::printf("example2-2: %s -ds example1.dat-s -o example2.result -p param.sdpa\n", argv0);
    std::printf("example2-3: %s -ds example1.dat-s -o example3.result -pt 2\n", argv0);
}

bool ends_with_s(const char *f) {
    size_t n = std::strlen(f);
    return n >= 2 && f[n - 1] == 's' && f[n - 2] == '-';
}

int pt_type(const char *s) {
    int t = std::atoi(s);
    return (t == 1 || t == 2) ? t : 0;
}

} // namespace

extern "C" int sddd_cli_main(int argc, char **argv) {
    std::setbuf(stdout, nullptr);
    time_t ltime;
    std::time(&ltime);
    std::printf("SDPA-DD start at    %s", std::ctime(&ltime));
    bool isInitFile = false, isInitSparse = false, isDataSparse = false;
    const char *dataFile = nullptr, *initFile = nullptr, *outFile = nullptr, *paraFile = nullptr;
    const char *pointFile = nullptr; // -wd / -ws: the final point as an init file (this build's extension)
    bool isPointSparse = false;
    int ptype = 0;
    double kappa = 1.2;
    int device = 0;
    if (const char *d = std::getenv("SDDD_DEVICE")) device = std::atoi(d);
    int tc_slices = 0; // tensor-core split Cholesky of B (this build's extension)
    if (const char *s = std::getenv("SDDD_TC_SLICES")) tc_slices = std::atoi(s);
    if (argc == 1) {
        usage(argv[0]);
        return 1;
    }
    if (argv[1][0] == '-') {
        for (int i = 0; i < argc; ++i) {
            const char *t = argv[i];
            if (!std::strcmp(t, "-dd") && i + 1 < argc) {
                dataFile = argv[++i];
            } else if (!std::strcmp(t, "-ds") && i + 1 < argc) {
                dataFile = argv[++i];
                isDataSparse = true;
            } else if ((!std::strcmp(t, "-id") || !std::strcmp(t, "-is")) && i + 1 < argc) {
                isInitSparse = !std::strcmp(t, "-is");
                initFile = argv[++i];
                isInitFile = true;
            } else if (!std::strcmp(t, "-o") && i + 1 < argc) {
                outFile = argv[++i];
            } else if (!std::strcmp(t, "-p") && i + 1 < argc) {
                paraFile = argv[++i];
            } else if (!std::strcmp(t, "-k") && i + 1 < argc) {
                kappa = std::atof(argv[++i]);
                std::printf("Kappa = %g\n", kappa);
            } else if (!std::strcmp(t, "-pt") && i + 1 < argc) {
                ptype = pt_type(argv[++i]);
                paraFile = nullptr;
            } else if (!std::strcmp(t, "-tc") && i + 1 < argc) {
                tc_slices = std::atoi(argv[++i]);
            } else if ((!std::strcmp(t, "-wd") || !std::strcmp(t, "-ws")) && i + 1 < argc) {
                isPointSparse = !std::strcmp(t, "-ws");
                pointFile = argv[++i];
            }
        }
    } else {
        dataFile = argv[1];
        isDataSparse = ends_with_s(dataFile);
        outFile = argc > 2 ? argv[2] : nullptr;
        paraFile = "./param.sdpa";
        for (int i = 3; i < argc; ++i) {
            if (!std::strcmp(argv[i], "-pt") && i + 1 < argc) {
                ptype = pt_type(argv[++i]);
                paraFile = nullptr;
            } else {
                initFile = argv[i];
                isInitFile = true;
                isInitSparse = ends_with_s(initFile);
            }
        }
    }
    if (!dataFile || !outFile) {
        usage(argv[0]);
        return 1;
    }
    std::printf("data      is %s : %s\n", dataFile, isDataSparse ? "sparse" : "dense");
    if (paraFile) std::printf("parameter is %s\n", paraFile);
    std::printf("out       is %s\n", outFile);
    if (initFile) std::printf("initial   is %s\n", initFile);
    else std::printf("\n");
    if (!paraFile) std::printf("set       is %s\n", ptype == 0 ? "DEFAULT" : ptype == 1 ? "UNSTABLE_BUT_FAST" : "STABLE_BUT_SLOW");
    // pinpal
    const auto t0 = std::chrono::steady_clock::now();
    FILE *fo = std::fopen(outFile, "w");
    if (!fo) {
        std::printf("Cannot open out file %s\n", outFile);
        return 0;
    }
    sddd::Param param = sddd::default_param(ptype);
    try {
        if (paraFile) param = sddd::read_param(paraFile);
    } catch (const sddd::Error &) {
        std::printf("Cannot open parameter file %s \n", paraFile);
        return 0;
    }
    std::fprintf(fo, "SDPA-DD start at %s", std::ctime(&ltime));
    sddd_ctx *ctx = nullptr;
    int rc = sddd_create(device, &ctx);
    if (rc != SDDD_OK) {
        std::fprintf(stderr, "%s\n", sddd_last_error(nullptr));
        return 1;
    }
    if (tc_slices != 0 && sddd_set_tc_split(ctx, tc_slices) != SDDD_OK) {
        std::fprintf(stderr, "%s\n", sddd_last_error(ctx));
        sddd_destroy(ctx);
        return 1;
    }
    struct Closer {
        sddd_ctx *c;
        ~Closer() { sddd_destroy(c); }
    } closer{ctx};
    sddd::Problem prob;
    try {
        prob = sddd::read_problem(dataFile, isDataSparse);
    } catch (const sddd::Error &e) {
        std::printf("%s\n", e.what());
        return 0;
    }
    for (auto &cm : prob.comments) std::fprintf(fo, "%s\n", cm.c_str());
    std::fprintf(fo, "data      is %s\n", dataFile);
    if (paraFile) std::fprintf(fo, "parameter is %s\n", paraFile);
    if (initFile) std::fprintf(fo, "initial   is %s\n", initFile);
    std::fprintf(fo, "out       is %s\n", outFile);
    try {
        sddd::finalize_problem(prob, kappa);
        sddd_attach_problem(ctx, std::move(prob));
    } catch (const sddd::Error &e) {
        std::printf("%s\n", e.what());
        std::fclose(fo);
        return 1;
    }
    if (isInitFile && sddd_read_initial_point(ctx, initFile, isInitSparse ? 1 : 0, param.lambdaStar) != SDDD_OK) {
        std::printf("%s\n", sddd_last_error(ctx));
        std::fclose(fo);
        return 1;
    }
    // Newton::initialize_bMat's report (sdpa_newton.cpp:345-391)
    sddd_schur_info form{};
    if (sddd_schur_form(ctx, &form, nullptr, nullptr, nullptr) == SDDD_OK && form.sparse) {
        std::printf("SPARSE computation\n");
        std::fprintf(fo, "SPARSE computation\n");
    } else {
        std::printf("DENSE computations\n");
        std::fprintf(fo, "DENSE computation\n");
    }
    const double fileRead = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    sddd_param p;
    p.maxIteration = param.maxIteration;
    p.epsilonStar = param.epsilonStar;
    p.lambdaStar = param.lambdaStar;
    p.omegaStar = param.omegaStar;
    p.lowerBound = param.lowerBound;
    p.upperBound = param.upperBound;
    p.betaStar = param.betaStar;
    p.betaBar = param.betaBar;
    p.gammaStar = param.gammaStar;
    p.epsilonDash = param.epsilonDash;
    double mainLoop = 0;
    rc = sddd_solve_stream(ctx, &p, stdout, fo, fileRead, &mainLoop);
    const double total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rc != SDDD_OK) std::fprintf(stderr, "%s\n", sddd_last_error(ctx));
    if (rc == SDDD_OK && pointFile && sddd_write_point(ctx, pointFile, isPointSparse ? 1 : 0) != SDDD_OK) {
        std::fprintf(stderr, "%s\n", sddd_last_error(ctx));
        rc = 1;
    }
    std::printf("  main loop time = %.6f\n", mainLoop);
    std::fprintf(fo, "    main loop time = %.6f\n", mainLoop);
    std::printf("      total time = %.6f\n", total);
    std::fprintf(fo, "        total time = %.6f\n", total);
    std::printf("file   read time = %.6f\n", fileRead);
    std::fprintf(fo, "  file   read time = %.6f\n", fileRead);
    std::fclose(fo);
    return rc == SDDD_OK ? 0 : 1;
}
