// ocean3d5_b200 <namelist>: drop-in executable for the reference's backend
// protocol (tools/compare_backends3d5.py:71 runs `binary nml`). All work is in
// the library call oc_run_namelist.
#include <cstdio>

#include "ocean_b200.h"

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: ocean3d5_b200 <namelist>\n");
        return 1;
    }
    return oc_run_namelist(argv[1]);
}
