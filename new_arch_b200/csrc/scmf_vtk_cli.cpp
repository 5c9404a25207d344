// scmf_vtk: drop-in for the reference's vtk.c converter (vtk.c:4-81).
//   scmf_vtk                 pha.dat -> out.vtk
//   scmf_vtk IN              IN -> out.vtk
//   scmf_vtk IN OUT          IN -> OUT
//   scmf_vtk IN OUT auto     per-point value count taken from the file instead
//                            of vtk.c's fixed six
#include <cstdio>
#include <cstring>

#include "scmf.h"

int main(int argc, char** argv) {
    const char* in = "pha.dat";
    const char* out = "out.vtk";
    if (argc >= 2) in = argv[1];
    if (argc >= 3) out = argv[2];
    const int vpp = (argc >= 4 && strcmp(argv[3], "auto") == 0) ? 0 : 6;
    printf("%d\n", argc);
    if (scmf_vtk_convert(in, out, vpp) != SCMF_OK) {
        fprintf(stderr, "ERROR: %s\n", scmf_last_error());
        return 1;
    }
    return 0;
}
