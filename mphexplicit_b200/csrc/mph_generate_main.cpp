// mph_generate — drop-in for the reference's pre-processor GeneratorForMph
// (generator/generator.cpp:37-47): `mph_generate [stem]` reads <stem>.boid
// and writes <stem>.grid (stem "sample" when none is given).  Unlike the
// reference it reports malformed input and exits non-zero.
#include <cstdio>
#include <string>

#include "mph_b200.h"

int main(int argc, char** argv) {
    const std::string stem = argc > 1 ? argv[1] : "sample";
    const std::string boid = stem + ".boid", grid = stem + ".grid";
    long long n = 0;
    const int st = mph_generate_grid_file(boid.c_str(), grid.c_str(), &n);
    if (st != MPH_OK) {
        char msg[512];
        mph_generator_last_error(msg, sizeof(msg));
        std::fprintf(stderr, "mph_generate: %s: %s (status %d)\n", boid.c_str(), msg, st);
        return 1;
    }
    std::fprintf(stderr, "%lld particles were generated\n", n);
    return 0;
}
