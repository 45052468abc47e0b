// Trace of the reference's ./fft_gkr program (TEST INFRASTRUCTURE).
//
// Compiles the unmodified reference source TruePix-main/Orion/Orion_nonzk/
// src/VPD/fft_circuit_GKR.cpp in place (its main renamed by the preprocessor)
// and runs the same steps as its main (:827-845) and engage_gkr (:770-825),
// one layer function at a time, printing what each step leaves behind:
//
//   layer <k> <size> <re im>...   circuit layer k (all layers when lg <= 6)
//   claim <stage> <re> <im>       alpha_beta_sum after V_output ("a0"),
//                                 addition_layer ("add"), mult_layer ("mult"),
//                                 intermediate_layer ("inter"), ifft_gkr ("ifft")
//   final <a.re a.im b.re b.im> x3   V_mult_add[0], addV_array[0], add_mult_sum[0]
//                                 after the last sumcheck round
//   result <0|1>                  every sumcheck and closing check passed
//   proof_size <bytes>            the reference's count (extension_gkr included)
//
// Usage: fft_gkr_harness <lg>. The randomness is the reference's: glibc rand()
// in its unseeded state, drawn in main's and engage_gkr's order.
#include <cstdio>
#include <cstdlib>

#define main reference_fft_gkr_main
#include "src/VPD/fft_circuit_GKR.cpp"
#undef main

static void put(const char* tag, const prime_field::field_element& x)
{
    printf("claim %s %llu %llu\n", tag, (unsigned long long)x.real, (unsigned long long)x.img);
}

static void put_lp(const linear_poly& p)
{
    printf(" %llu %llu %llu %llu", (unsigned long long)p.a.real, (unsigned long long)p.a.img,
           (unsigned long long)p.b.real, (unsigned long long)p.b.img);
}

int main(int argc, char* argv[])
{
    if (argc < 2) {
        fprintf(stderr, "usage: %s <lg>\n", argv[0]);
        return 2;
    }
    const int lg_size = atoi(argv[1]);
    prime_field::init();
    prime_field::init_random();
    init_array(lg_size + 6);
    prime_field::field_element* r = new prime_field::field_element[lg_size];
    for (int i = 0; i < lg_size; ++i) r[i] = prime_field::random();
    build_circuit(lg_size, r);
    if (lg_size <= 6) {
        for (size_t k = 0; k < C.circuit_val.size(); ++k) {
            printf("layer %zu %d", k, C.size[k]);
            for (int i = 0; i < C.size[k]; ++i)
                printf(" %llu %llu", (unsigned long long)C.circuit_val[k][i].real,
                       (unsigned long long)C.circuit_val[k][i].img);
            printf("\n");
        }
    }

    // engage_gkr's body, one step at a time
    alpha = prime_field::field_element(1);
    beta = prime_field::field_element(0);
    const int n = lg_size + 10;
    prime_field::field_element *r_0 = new prime_field::field_element[n], *omr_0 = new prime_field::field_element[n];
    prime_field::field_element *r_1 = new prime_field::field_element[n], *omr_1 = new prime_field::field_element[n];
    prime_field::field_element *r_u = new prime_field::field_element[n], *omr_u = new prime_field::field_element[n];
    prime_field::field_element *r_v = new prime_field::field_element[n], *omr_v = new prime_field::field_element[n];
    refresh_randomness(r_0, omr_0, n);
    refresh_randomness(r_1, omr_1, n);
    const size_t L = C.circuit_val.size();
    prime_field::field_element s = V_output(omr_0, r_0, C.circuit_val[L - 1], mylog(C.size[L - 1]), C.size[L - 1]);
    put("a0", s);
    bool ok = true;
    ok &= addition_layer(s, C.circuit_val[L - 2], C.size[L - 2] / 64, 64, r_0, omr_0, r_1, omr_1, r_u, omr_u, r_v,
                         omr_v);
    put("add", s);
    ok &= mult_layer(s, C.circuit_val[L - 3], C.size[L - 3], 64, r_0, omr_0, r_1, omr_1, r_u, omr_u, r_v, omr_v);
    put("mult", s);
    ok &= intermediate_layer(s, C.circuit_val[L - 4], C.size[L - 4], r_0, omr_0, r_1, omr_1, r_u, omr_u, r_v, omr_v);
    put("inter", s);
    ok &= ifft_gkr(s, C.size[L - 4], r_0, omr_0, r_1, omr_1, r_u, omr_u, r_v, omr_v);
    put("ifft", s);
    ok &= extension_gkr(s, C.size[L - 4], r_0, omr_0, r_1, omr_1, r_u, omr_u, r_v, omr_v);
    printf("final");
    put_lp(V_mult_add[0]);
    put_lp(addV_array[0]);
    put_lp(add_mult_sum[0]);
    printf("\nresult %d\nproof_size %d\n", ok ? 1 : 0, proof_size);
    return 0;
}
