// A caller of the reference's C++ API ("Falcons/api/falcons.hpp"), built twice by
// tests/native/Makefile: against include/dropin (the B200 library behind include/falcons_gpu.hpp,
// with the reference's own Falcons::Config) as _build/dropin_api, and against the reference's
// header itself as _build/dropin_api_ref, so that the tests compare the two builds' answers.
// Each command exercises one part of the API (run as a child process by tests/test_dropin_cpu.py
// and tests/test_dropin_gpu.py):
//   config    <file>        Falcons_read_config on a stream file: prints the Config fields
//   bound     N d0 [d1..]   Falcons_compress_size_bound<float/double> for those dims
//   roundtrip <in.f32> <out.stream> <out.f32> d0 [d1..] <abs_eb>
//                           Falcons_compress<float> (ALGO_INTERP_LORENZO, EB_ABS) then
//                           Falcons_decompress<float>; writes the stream and the reconstruction
//   decompress <stream> <out.f32>
//                           Falcons_decompress<float> of a stream file into a caller buffer of
//                           the stream's size (the capacity overload)
//   integral                an int32 compress: must throw std::invalid_argument
// Test infrastructure; the product never builds it.
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <vector>

#include "Falcons/api/falcons.hpp"

static std::vector<char> slurp(const char *path) {
    std::ifstream f(path, std::ios::binary);
    return std::vector<char>((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
}

static void print_config(const Falcons::Config &c) {
    printf("N=%d num=%zu", (int)c.N, c.num);
    for (size_t d : c.dims) printf(" dim=%zu", d);
    printf(" cmprAlgo=%d errorBoundMode=%d absErrorBound=%.17g relErrorBound=%.17g quantbinCnt=%d blockSize=%d "
           "interpAlgo=%d interpDirection=%d interpAnchorStride=%d interpAlpha=%.17g interpBeta=%.17g openmp=%d "
           "lorenzo=%d lorenzo2=%d regression=%d regression2=%d\n",
           (int)c.cmprAlgo, (int)c.errorBoundMode, c.absErrorBound, c.relErrorBound, c.quantbinCnt, c.blockSize,
           (int)c.interpAlgo, (int)c.interpDirection, c.interpAnchorStride, c.interpAlpha, c.interpBeta, (int)c.openmp,
           (int)c.lorenzo, (int)c.lorenzo2, (int)c.regression, (int)c.regression2);
}

int main(int argc, char **argv) {
    if (argc < 2) return 2;
    try {
        const std::string cmd = argv[1];
        if (cmd == "config") {
            const std::vector<char> s = slurp(argv[2]);
            Falcons::Config c;
            Falcons_read_config(c, s.data(), s.size());
            print_config(c);
            return 0;
        }
        if (cmd == "bound") {
            std::vector<size_t> d;
            for (int i = 3; i < argc; i++) d.push_back((size_t)atoll(argv[i]));
            Falcons::Config c;
            c.setDims(d.begin(), d.end());
            printf("%zu %zu\n", Falcons::Falcons_compress_size_bound<float>(c),
                   Falcons::Falcons_compress_size_bound<double>(c));
            return 0;
        }
        if (cmd == "roundtrip") {
            std::vector<size_t> d;
            for (int i = 5; i < argc - 1; i++) d.push_back((size_t)atoll(argv[i]));
            Falcons::Config c;
            c.setDims(d.begin(), d.end());
            c.cmprAlgo = Falcons::ALGO_INTERP_LORENZO;
            c.errorBoundMode = Falcons::EB_ABS;
            c.absErrorBound = atof(argv[argc - 1]);
            std::vector<float> x(c.num);
            FILE *f = fopen(argv[2], "rb");
            if (!f || fread(x.data(), 4, c.num, f) != c.num) return 3;
            fclose(f);
            size_t n = 0;
            char *s = Falcons_compress<float>(c, x.data(), n);
            Falcons::writefile(argv[3], s, n);
            Falcons::Config c2;
            float *y = Falcons_decompress<float>(c2, s, n);
            Falcons::writefile(argv[4], y, c2.num);
            print_config(c2);
            delete[] s;
            delete[] y;
            return 0;
        }
        if (cmd == "decompress") {
            const std::vector<char> s = slurp(argv[2]);
            Falcons::Config c;
            Falcons_read_config(c, s.data(), s.size());
            std::vector<float> y(c.num);
            float *p = y.data();
            Falcons_decompress<float>(c, s.data(), s.size(), p, y.size());
            Falcons::writefile(argv[3], y.data(), c.num);
            print_config(c);
            return 0;
        }
        if (cmd == "integral") {
            Falcons::Config c(10, 10);
            std::vector<int32_t> x(100, 7);
            size_t n = 0;
            try {
                char *s = Falcons_compress<int32_t>(c, x.data(), n);
                delete[] s;
            } catch (const std::invalid_argument &e) {
                printf("invalid_argument: %s\n", e.what());
                return 0;
            }
            return 4;
        }
    } catch (const std::invalid_argument &e) {
        printf("invalid_argument: %s\n", e.what());
        return 5;
    } catch (const std::exception &e) {
        printf("exception: %s\n", e.what());
        return 6;
    }
    return 2;
}
