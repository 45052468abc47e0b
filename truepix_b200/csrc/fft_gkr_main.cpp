// ./fft_gkr <lg> <outfile> [trace]: the program Orion's polynomial-commitment
// verifier runs from its working directory (TruePix-main/Orion/Orion_nonzk/
// src/VPD/vpd_verifier.cpp:80-89), with the proof made on the device by
// tp_fft_gkr. Writes "v_time proof_size p_time" as "%f %d %f\n" to <outfile>
// (src/VPD/fft_circuit_GKR.cpp:827-845) and reports a failed check on stderr as
// the reference does; the optional third argument names a trace file.
#include <cstdio>

#include "native_fp2.h"
#include "orion_gpu.h"

int main(int argc, char* argv[])
{
    int lg = 0;
    if (argc < 3 || sscanf(argv[1], "%d", &lg) != 1) {
        fprintf(stderr, "usage: %s <lg> <outfile> [trace]\n", argv[0]);
        return 1;
    }
    double v_time = 0, p_time = 0;
    long long proof_size = 0;
    int accepted = 0;
    if (tp_fft_gkr(lg, &v_time, &proof_size, &p_time, &accepted, argc > 3 ? argv[3] : nullptr) != 0) {
        fprintf(stderr, "fft_gkr: %s\n", tp_last_error());
        return 1;
    }
    if (!accepted) fprintf(stderr, "Error, fft gkr failed\n");
    FILE* out = fopen(argv[2], "w");
    if (!out) {
        fprintf(stderr, "fft_gkr: cannot write %s\n", argv[2]);
        return 1;
    }
    fprintf(out, "%f %d %f\n", (float)v_time, (int)proof_size, (float)p_time);
    fclose(out);
    return 0;
}
