// C entry points over the reference's zero-knowledge Orion sources (TEST
// INFRASTRUCTURE).
//
// Compiled by `make -C oracle ref` together with the unmodified reference files
// under TruePix-main/Orion/Orion_zk (compiled in place) into
// oracle/_ref/liborion_zk_ref.so. The golden generator calls these; the shipped
// library never links them.
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "VPD/linearPC.h"
#include "linear_code/linear_code_encode.h"
#include "linear_gkr/prime_field.h"
#include "truepix/truepix_gkr.h"

extern "C" {

// The commit phase of linearPC_multi_commit_zk
// (examples/multivariate_PC_test_commit.cpp:280-340) on a frame given as its
// TruePix-layout coefficients (n_copies_padded * 512 elements {img, real}, as
// load_coefs leaves them): layout, alloc_masked_from_seed /
// alloc_mask_from_seed with `seed`, expander_init in the default glibc rand()
// state, commit_pair. Writes both roots (hex form too) and, when mask_out is
// set, the mask polynomial. Call once per process: the reference keeps encoder
// state.
int ref_zk_commit(const uint64_t* coefs, int copies, int copy_size, int const_idx, int const_val,
                  unsigned long long seed, unsigned char* root_masked, unsigned char* root_mask,
                  char* hex_masked, char* hex_mask, uint64_t* mask_out)
{
    typedef prime_field::field_element F;
    prime_field::init();
    truepix::Layout lay;
    lay.copies = copies;
    lay.copy_size = copy_size;
    lay.const_idx = const_idx;
    lay.const_val = const_val;
    lay.padded_copies = truepix::next_pow2_int(copies);
    lay.n = (long long)lay.padded_copies * lay.padded_copy_size;
    lay.lg_n = 0;
    while ((1LL << lay.lg_n) < lay.n) lay.lg_n++;
    srand(1);
    expander_init(lay.n / column_size);
    const F* c = reinterpret_cast<const F*>(coefs);
    F* masked = truepix::alloc_masked_from_seed(c, lay, seed);
    F* mask = truepix::alloc_mask_from_seed(lay, seed);
    if (mask_out) memcpy(mask_out, mask, 16 * (size_t)lay.n);
    set_retain_encoded_codeword(true);
    zk_pair_commit pc = commit_pair(masked, mask, lay.n);
    memcpy(root_masked, &pc.mt_masked[1], 32);
    memcpy(root_mask, &pc.mt_mask[1], 32);
    memcpy(hex_masked, truepix::root_hex(pc.mt_masked[1]).c_str(), 65);
    memcpy(hex_mask, truepix::root_hex(pc.mt_mask[1]).c_str(), 65);
    delete[] masked;
    delete[] mask;
    return 0;
}

}  // extern "C"
