// linearPC_multi_{commit,prove,open}[_zk] <copies> <userandom>
//
// The six Orion programs TruePix runs as subprocesses
// (TruePix-main/Orion/Orion_nonzk/examples/multivariate_PC_test_{commit,prove,open}.cpp
// and the zero-knowledge Orion_zk ones, called through
// libTruePix/fp2_link.py:639-651 and run_truepix_prover.py:379-398), over this
// library: the commits, the openings and the openings' checks run on the
// device. One source, built once per program (TP_CLI_PHASE 1 commit, 2 prove,
// 3 open; TP_CLI_ZK 1 for the zero-knowledge commit pair: the masked polynomial
// and the mask from a seed file, opened over the even and the odd columns). The
// process contract is the reference's:
//
//   arguments    <copies> <userandom>; userandom must be 0 (input.txt)
//   environment  TRUEPIX_PROTOCOL (fp2-linked-v1 or truepix), TRUEPIX_COPY_SIZE,
//                TRUEPIX_CONST_IDX, TRUEPIX_CONST_VAL, TRUEPIX_ORION_COMMIT_FILE,
//                TRUEPIX_GKR_POINT_FILE, TRUEPIX_ORION_MODE, TRUEPIX_ORION_RESULT_FILE,
//                TRUEPIX_MASK_SEED_FILE
//   files        input.txt (one copy per line), orion_commit.json (the manifest,
//                include/truepix/truepix_gkr.h:391-418), the GKR point file
//                ("<count>" then "<real> <imag>" per coordinate), orion_proof.bin
//                or orion_proof_masked.bin + orion_proof_mask.bin
//                (src/truepix/orion_proof.cpp:67-95), orion_mask_seed.txt
//   stdout       the lines fp2_link.py parses: "Commit time", "Open time",
//                "Proof size for tensor IOP ... bytes", "Verification time"
//   exit status  0 when every check passed
//
// Only the TruePix protocol's NIZK path is served: the legacy Y/Cb/Cr benchmark
// packing (TRUEPIX_PROTOCOL unset) and the interactive Orion mode are refused
// with a message.
//
// EC(y1): the reference's prover and verifier both re-run a GKR proof of the
// code of the combined message (generate_circuit + zk_verifier::verify,
// src/VPD/linearPC.cpp:585-605 and :851-861) in-process; its outcome gates the
// opening. Here the check is the statement that GKR proves, evaluated directly
// on the device: Enc(combined_message) equals the combined codeword at the
// second batch of transcript-drawn positions (the assertion of :604-605).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "native_fp2.h"
#include "orion_gpu.h"

#ifndef TP_CLI_PHASE
#error "TP_CLI_PHASE must be 1 (commit), 2 (prove) or 3 (open)"
#endif
#ifndef TP_CLI_ZK
#define TP_CLI_ZK 0
#endif

namespace {

typedef uint64_t u64;
constexpr u64 P61 = 0x1FFFFFFFFFFFFFFFull;
constexpr int kColumns = 128;         // column_size (include/linear_code/parameter.h)
constexpr int kPaddedCopy = 512;
constexpr double kTargetDistance = 0.07;
const char* const kProtocol = "fp2-linked-v1";
const char* const kProtocolAlias = "truepix";
const char* const kLayoutId = "copy-major-384-const128-pad512-v1";

double now() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }
int query_count() { return (int)(-128 / std::log2(1 - kTargetDistance)); }   // linearPC.cpp:440

std::string env_or(const char* name, const char* fallback)
{
    const char* e = getenv(name);
    return (e && *e) ? std::string(e) : std::string(fallback);
}
bool protocol_ok(const std::string& p) { return p == kProtocol || p == kProtocolAlias; }

// ---- layout (truepix_gkr.h:87-153) ----------------------------------------------
struct Layout {
    int copies = 0, padded_copies = 0, copy_size = 384, padded_copy_size = kPaddedCopy, const_idx = 384,
        const_val = 128;
    long long n = 0;
    int lg_n = 0;
    bool operator==(const Layout& o) const
    {
        return copies == o.copies && padded_copies == o.padded_copies && copy_size == o.copy_size &&
               padded_copy_size == o.padded_copy_size && const_idx == o.const_idx && const_val == o.const_val &&
               n == o.n && lg_n == o.lg_n;
    }
};

bool parse_args(int argc, char** argv, int& copies, int& userandom)
{
    if (argc < 3) {
        fprintf(stderr, "usage: %s <copies> <userandom>\n", argv[0]);
        return false;
    }
    if (sscanf(argv[1], "%d", &copies) != 1 || copies <= 0) {
        fprintf(stderr, "invalid copies '%s': expected a positive integer\n", argv[1]);
        return false;
    }
    if (sscanf(argv[2], "%d", &userandom) != 1 || (userandom != 0 && userandom != 1)) {
        fprintf(stderr, "invalid userandom '%s': expected 0 or 1\n", argv[2]);
        return false;
    }
    return true;
}

bool make_layout(int copies, Layout& L)
{
    L = Layout();
    L.copies = copies;
    if (const char* e = getenv("TRUEPIX_COPY_SIZE")) L.copy_size = atoi(e);
    if (const char* e = getenv("TRUEPIX_CONST_IDX")) L.const_idx = atoi(e);
    if (const char* e = getenv("TRUEPIX_CONST_VAL")) L.const_val = atoi(e);
    if (L.copy_size <= 0 || L.copy_size > L.padded_copy_size) {
        fprintf(stderr, "TruePix: invalid TRUEPIX_COPY_SIZE=%d (padded copy is %d)\n", L.copy_size,
                L.padded_copy_size);
        return false;
    }
    if (L.const_idx >= L.padded_copy_size) {
        fprintf(stderr, "TruePix: TRUEPIX_CONST_IDX=%d out of range\n", L.const_idx);
        return false;
    }
    if (L.const_idx >= 0 && L.const_idx < L.copy_size) {
        fprintf(stderr, "TruePix: TRUEPIX_CONST_IDX=%d overlaps the %d values read from input.txt; GKR and Orion "
                        "would pack different polynomials\n", L.const_idx, L.copy_size);
        return false;
    }
    L.padded_copies = 1;
    while (L.padded_copies < copies) L.padded_copies <<= 1;
    L.n = (long long)L.padded_copies * L.padded_copy_size;
    while ((1LL << L.lg_n) < L.n) L.lg_n++;
    return true;
}

// ---- input.txt (truepix_gkr.h:155-206) --------------------------------------------
// the private values, copy-major (copies x copy_size), reduced mod p; `small`
// when every value and the constant fit a byte (then the commit reads bytes)
struct Input {
    std::vector<u64> vals;
    bool small = true;
};

bool load_input(const char* path, const Layout& L, Input& in)
{
    std::ifstream f(path);
    if (!f) {
        fprintf(stderr, "TruePix: cannot open %s for reading\n", path);
        return false;
    }
    in.vals.assign((size_t)L.copies * L.copy_size, 0);
    in.small = L.const_val >= 0 && L.const_val < 256;
    std::string line;
    int copy = 0;
    while (copy < L.copies && std::getline(f, line)) {
        std::istringstream iss(line);
        long long v;
        int filled = 0;
        while (filled < L.copy_size && iss >> v) {
            if (v < 0) {
                fprintf(stderr, "TruePix: negative value on line %d of %s\n", copy + 1, path);
                return false;
            }
            const u64 x = (u64)v % P61;
            if (x > 255) in.small = false;
            in.vals[(size_t)copy * L.copy_size + filled++] = x;
        }
        if (filled != L.copy_size) {
            fprintf(stderr, "TruePix: copy %d has %d values, expected %d\n", copy, filled, L.copy_size);
            return false;
        }
        ++copy;
    }
    if (copy < L.copies) {
        fprintf(stderr, "TruePix: %s has %d lines, expected %d\n", path, copy, L.copies);
        return false;
    }
    printf("TruePix layout: C=%d padded_copies=%d N=%lld lg_N=%d copy_size=%d const[%d]=%d\n", L.copies,
           L.padded_copies, L.n, L.lg_n, L.copy_size, L.const_idx, L.const_val);
    return true;
}

// ---- GKR point (truepix_gkr.h:231-276): (real, imag) pairs ----------------------------
bool load_point(int lg_n, std::vector<u64>& pt)
{
    const char* env = getenv("TRUEPIX_GKR_POINT_FILE");
    if (!env) {
        fprintf(stderr, "TruePix: TRUEPIX_GKR_POINT_FILE is not set\n");
        return false;
    }
    std::string p(env);
    if (p.size() >= 5 && p.compare(p.size() - 5, 5, ".json") == 0)
        p = p.substr(0, p.size() - 5) + ".txt";
    else if (p.size() < 4 || p.compare(p.size() - 4, 4, ".txt") != 0)
        p += ".txt";
    std::ifstream f(p);
    if (!f) {
        fprintf(stderr, "TruePix: cannot open GKR point file %s\n", p.c_str());
        return false;
    }
    int k = 0;
    if (!(f >> k) || k != lg_n) {
        fprintf(stderr, "TruePix: GKR point has %d coordinates, expected %d\n", k, lg_n);
        return false;
    }
    pt.assign(2 * (size_t)lg_n, 0);
    for (int i = 0; i < lg_n; ++i) {
        unsigned long long re = 0, im = 0;
        if (!(f >> re >> im)) {
            fprintf(stderr, "TruePix: GKR point file %s truncated at %d\n", p.c_str(), i);
            return false;
        }
        if (re >= P61 || im >= P61) {
            fprintf(stderr, "TruePix: GKR point coordinate %d is not reduced\n", i);
            return false;
        }
        pt[2 * i] = re;
        pt[2 * i + 1] = im;
    }
    printf("TruePix: loaded GKR point from %s\n", p.c_str());
    return true;
}

// ---- manifest (truepix_gkr.h:366-516) ---------------------------------------------
// root_hex: the digest's little-endian 64-bit words 1, 0, 3, 2 as %016llx
std::string root_hex(const unsigned char* d)
{
    char buf[65];
    const int order[4] = {1, 0, 3, 2};
    for (int i = 0; i < 4; ++i) {
        u64 w = 0;
        memcpy(&w, d + 8 * order[i], 8);
        snprintf(buf + 16 * i, 17, "%016llx", (unsigned long long)w);
    }
    return std::string(buf, 64);
}

bool root_from_hex(const std::string& hex, unsigned char* d)
{
    if (hex.size() != 64) return false;
    const int order[4] = {1, 0, 3, 2};
    for (int i = 0; i < 4; ++i) {
        char buf[17];
        memcpy(buf, hex.data() + 16 * i, 16);
        buf[16] = 0;
        char* end = nullptr;
        const u64 w = strtoull(buf, &end, 16);
        if (end != buf + 16) return false;
        memcpy(d + 8 * order[i], &w, 8);
    }
    return true;
}

std::string manifest_path() { return env_or("TRUEPIX_ORION_COMMIT_FILE", "orion_commit.json"); }

bool write_manifest(const Layout& L, const std::string& root, const std::string& mask_root, bool zk)
{
    const std::string path = manifest_path();
    FILE* f = fopen(path.c_str(), "w");
    if (!f) {
        fprintf(stderr, "TruePix: cannot write commit manifest %s\n", path.c_str());
        return false;
    }
    const char* e = getenv("TRUEPIX_PROTOCOL");
    fprintf(f, "{\n  \"protocol\": \"%s\",\n  \"layout\": \"%s\",\n  \"zk\": %s,\n  \"copies\": %d,\n"
               "  \"padded_copies\": %d,\n  \"copy_size\": %d,\n  \"padded_copy_size\": %d,\n  \"const_idx\": %d,\n"
               "  \"const_val\": %d,\n  \"n\": %lld,\n  \"lg_n\": %d,\n  \"masked_root\": \"%s\",\n"
               "  \"mask_root\": \"%s\"\n}\n",
            (e && protocol_ok(e)) ? e : kProtocol, kLayoutId, zk ? "true" : "false", L.copies, L.padded_copies,
            L.copy_size, L.padded_copy_size, L.const_idx, L.const_val, L.n, L.lg_n, root.c_str(), mask_root.c_str());
    fclose(f);
    printf("TruePix: wrote commit manifest %s (zk=%s masked_root=%s mask_root=%s)\n", path.c_str(),
           zk ? "true" : "false", root.c_str(), mask_root.c_str());
    return true;
}

// ---- the mask seed (Orion_zk include/truepix/truepix_gkr.h:294-329) ---------------
std::string mask_seed_path() { return env_or("TRUEPIX_MASK_SEED_FILE", "orion_mask_seed.txt"); }

bool mask_seed_read(u64& seed)
{
    std::ifstream in(mask_seed_path());
    if (!in) {
        fprintf(stderr, "TruePix: cannot open mask seed file %s; run the commit phase (run_fennel_signer.py) first\n",
                mask_seed_path().c_str());
        return false;
    }
    unsigned long long v = 0;
    if (!(in >> v)) {
        fprintf(stderr, "TruePix: malformed mask seed file %s\n", mask_seed_path().c_str());
        return false;
    }
    seed = v;
    return true;
}

bool mask_seed_create(u64& seed)
{
    std::ifstream urandom("/dev/urandom", std::ios::binary);
    unsigned long long v = 0;
    if (!urandom || !urandom.read(reinterpret_cast<char*>(&v), sizeof(v))) {
        fprintf(stderr, "TruePix: cannot read /dev/urandom for the mask seed\n");
        return false;
    }
    std::ofstream out(mask_seed_path(), std::ios::trunc);
    if (!out) {
        fprintf(stderr, "TruePix: cannot write mask seed file %s\n", mask_seed_path().c_str());
        return false;
    }
    out << v << "\n";
    seed = v;
    return true;
}

struct Manifest {
    Layout lay;
    std::string masked_root, mask_root;
    bool zk = true;
};

bool read_manifest(Manifest& m)
{
    const std::string path = manifest_path();
    std::ifstream f(path);
    if (!f) {
        fprintf(stderr, "TruePix: cannot open commit manifest %s; run the commit "
                        "phase (run_fennel_signer.py) first\n", path.c_str());
        return false;
    }
    const std::string body((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    auto value_at = [&](const char* key, size_t& pos) {
        const std::string pat = std::string("\"") + key + "\"";
        const size_t k = body.find(pat);
        if (k == std::string::npos) return false;
        pos = body.find(':', k + pat.size());
        return pos != std::string::npos;
    };
    auto str = [&](const char* key, std::string& out) {
        size_t c;
        if (!value_at(key, c)) return false;
        const size_t a = body.find('"', c), b = a == std::string::npos ? a : body.find('"', a + 1);
        if (b == std::string::npos) return false;
        out = body.substr(a + 1, b - a - 1);
        return true;
    };
    auto num = [&](const char* key, long long& out) {
        size_t c;
        if (!value_at(key, c)) return false;
        out = strtoll(body.c_str() + c + 1, nullptr, 10);
        return true;
    };
    std::string protocol, layout;
    long long v[10];
    const char* keys[10] = {"copies", "padded_copies", "copy_size", "padded_copy_size", "const_idx",
                            "const_val", "n", "lg_n", nullptr, nullptr};
    bool ok = str("protocol", protocol) && str("layout", layout) && str("masked_root", m.masked_root) &&
              str("mask_root", m.mask_root);
    for (int i = 0; ok && i < 8; ++i) ok = num(keys[i], v[i]);
    if (!ok) {
        fprintf(stderr, "TruePix: commit manifest %s is missing fields\n", path.c_str());
        return false;
    }
    size_t c;
    m.zk = true;
    if (value_at("zk", c)) {
        size_t p = c + 1;
        while (p < body.size() && (body[p] == ' ' || body[p] == '\t' || body[p] == '\n')) ++p;
        if (body.compare(p, 5, "false") == 0) m.zk = false;
    }
    if (!protocol_ok(protocol) || layout != kLayoutId) {
        fprintf(stderr, "TruePix: commit manifest %s has protocol=%s layout=%s\n", path.c_str(), protocol.c_str(),
                layout.c_str());
        return false;
    }
    m.lay.copies = (int)v[0];
    m.lay.padded_copies = (int)v[1];
    m.lay.copy_size = (int)v[2];
    m.lay.padded_copy_size = (int)v[3];
    m.lay.const_idx = (int)v[4];
    m.lay.const_val = (int)v[5];
    m.lay.n = v[6];
    m.lay.lg_n = (int)v[7];
    return true;
}

// ---- device plumbing --------------------------------------------------------------
struct Dev {
    void* p = nullptr;
    ~Dev() { if (p) cudaFree(p); }
    template <class T> T* as() const { return static_cast<T*>(p); }
};

bool cuda_ok(cudaError_t e, const char* what)
{
    if (e == cudaSuccess) return true;
    fprintf(stderr, "TruePix: %s: %s\n", what, cudaGetErrorString(e));
    return false;
}
bool lib_ok(int rc, const char* what)
{
    if (rc == 0) return true;
    fprintf(stderr, "TruePix: %s: %s\n", what, tp_last_error());
    return false;
}
bool alloc(Dev& d, size_t bytes) { return cuda_ok(cudaMalloc(&d.p, bytes ? bytes : 16), "device allocation"); }
bool upload(Dev& d, const void* h, size_t bytes)
{
    return alloc(d, bytes) && cuda_ok(cudaMemcpy(d.p, h, bytes, cudaMemcpyHostToDevice), "upload");
}
bool download(void* h, const void* d, size_t bytes)
{
    return cuda_ok(cudaMemcpy(h, d, bytes, cudaMemcpyDeviceToHost), "download");
}

// one committed polynomial: its row-major codeword and Merkle tree on the device
struct Poly {
    Dev rows, tree;
    unsigned char root[32];
};

struct Frame {
    Dev pixels, src;   // the frame's bytes, or (values above 255) its N-element vector {img, real}
    long long msg_len = 0, cw_len = 0, leaves = 0;
    Poly plain, masked, mask;
};

bool sizes(const Layout& L, Frame& F)
{
    F.msg_len = L.n / kColumns;
    F.cw_len = tp_orion_codeword_len(F.msg_len);
    F.leaves = tp_orion_tree_leaves(L.n);
    return (F.cw_len > 0 && F.leaves > 0) || lib_ok(-1, "codeword size");
}
bool alloc_poly(const Frame& F, Poly& P)
{
    return alloc(P.rows, 16 * (size_t)F.cw_len * kColumns) && alloc(P.tree, 64 * (size_t)F.leaves);
}
bool fetch_root(Poly& P) { return download(P.root, P.tree.as<unsigned char>() + 32, 32); }
bool upload_bytes(const Input& in, Frame& F)
{
    std::vector<unsigned char> b(in.vals.size());
    for (size_t i = 0; i < b.size(); ++i) b[i] = (unsigned char)in.vals[i];
    return upload(F.pixels, b.data(), b.size());
}

// commit(): the plain polynomial (truepix_gkr.h layout)
bool commit_frame(const Layout& L, const Input& in, Frame& F)
{
    if (!sizes(L, F) || !alloc_poly(F, F.plain)) return false;
    if (in.small) {
        if (!upload_bytes(in, F) ||
            !lib_ok(tp_orion_commit_pixels_dev(F.pixels.p, L.copies, L.padded_copies, L.copy_size,
                                               L.padded_copy_size, L.const_idx, (uint64_t)L.const_val,
                                               F.plain.rows.p, F.plain.tree.p, nullptr), "commit"))
            return false;
    } else {
        std::vector<u64> v(2 * (size_t)L.n, 0);   // {img, real} per element
        for (int c = 0; c < L.copies; ++c) {
            for (int w = 0; w < L.copy_size; ++w)
                v[2 * ((size_t)c * L.padded_copy_size + w) + 1] = in.vals[(size_t)c * L.copy_size + w];
            if (L.const_idx >= 0) v[2 * ((size_t)c * L.padded_copy_size + L.const_idx) + 1] = (u64)L.const_val % P61;
        }
        if (!upload(F.src, v.data(), 8 * v.size()) ||
            !lib_ok(tp_orion_commit_dev(F.src.p, L.n, F.plain.rows.p, F.plain.tree.p, nullptr), "commit"))
            return false;
    }
    return fetch_root(F.plain);
}

// commit_pair(): the masked polynomial and the mask from the seed (Orion_zk)
// splitmix64 (Steele, Lea and Flood's SplitMix generator, 64-bit output)
u64 splitmix64(u64& state)
{
    state += 0x9E3779B97F4A7C15ull;
    u64 z = state;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// commit_pair(): the masked polynomial and the mask from the seed (Orion_zk). Byte
// inputs are committed from their bytes (the library draws the mask on the
// device); other inputs from the two element vectors built here: the mask is zero
// except at the private wires (copy < copies, wire < copy_size), which take the
// seed's splitmix64 outputs mod p in flat order (real parts; Orion_zk
// include/truepix/truepix_gkr.h:339-362), and masked = frame + mask.
bool commit_frame_zk(const Layout& L, const Input& in, u64 seed, Frame& F)
{
    if (!sizes(L, F) || !alloc_poly(F, F.masked) || !alloc_poly(F, F.mask)) return false;
    if (in.small) {
        if (!upload_bytes(in, F)) return false;
        return lib_ok(tp_orion_commit_zk_pixels_dev(F.pixels.p, L.copies, L.padded_copies, L.copy_size,
                                                    L.padded_copy_size, L.const_idx, (uint64_t)L.const_val, seed,
                                                    F.masked.rows.p, F.masked.tree.p, F.mask.rows.p, F.mask.tree.p,
                                                    nullptr), "commit pair") &&
               fetch_root(F.masked) && fetch_root(F.mask);
    }
    std::vector<u64> masked(2 * (size_t)L.n, 0), mask(2 * (size_t)L.n, 0);   // {img, real} per element
    u64 state = seed;
    for (int c = 0; c < L.copies; ++c) {
        const size_t base = (size_t)c * L.padded_copy_size;
        for (int w = 0; w < L.copy_size; ++w) {
            const u64 m = splitmix64(state) % P61;
            const u64 x = in.vals[(size_t)c * L.copy_size + w];
            mask[2 * (base + w) + 1] = m;
            masked[2 * (base + w) + 1] = x + m >= P61 ? x + m - P61 : x + m;
        }
        if (L.const_idx >= 0) masked[2 * (base + L.const_idx) + 1] = (u64)L.const_val % P61;
    }
    Dev d_masked, d_mask;
    return upload(d_masked, masked.data(), 8 * masked.size()) && upload(d_mask, mask.data(), 8 * mask.size()) &&
           lib_ok(tp_orion_commit_dev(d_masked.p, L.n, F.masked.rows.p, F.masked.tree.p, nullptr), "commit") &&
           lib_ok(tp_orion_commit_dev(d_mask.p, L.n, F.mask.rows.p, F.mask.tree.p, nullptr), "commit") &&
           fetch_root(F.masked) && fetch_root(F.mask);
}

// the MLE of the frame's (plain) polynomial at the GKR point, LSB first
// (truepix::mle_gkr, truepix_gkr.h:210-229): out (real, imag)
bool frame_mle(const Layout& L, const Input& in, Frame& F, const std::vector<u64>& pt, u64 out[2])
{
    Dev z, o;
    if (!upload(z, pt.data(), 8 * pt.size()) || !alloc(o, 16)) return false;
    if (in.small) {
        if (!F.pixels.p && !upload_bytes(in, F)) return false;
        if (!lib_ok(tp_mle_eval_pixels(F.pixels.p, L.copies, L.padded_copies, L.copy_size, L.padded_copy_size,
                                       L.const_idx, (uint64_t)L.const_val, z.p, o.p, nullptr), "MLE"))
            return false;
    } else {
        std::vector<u64> x((size_t)L.n, 0);
        for (int c = 0; c < L.copies; ++c) {
            for (int w = 0; w < L.copy_size; ++w)
                x[(size_t)c * L.padded_copy_size + w] = in.vals[(size_t)c * L.copy_size + w];
            if (L.const_idx >= 0) x[(size_t)c * L.padded_copy_size + L.const_idx] = (u64)L.const_val % P61;
        }
        Dev dx;
        if (!upload(dx, x.data(), 8 * x.size()) ||
            !lib_ok(tp_mle_eval_base_dev(dx.p, z.p, L.lg_n, o.p, nullptr), "MLE"))
            return false;
    }
    return download(out, o.p, 16);
}

// r0 (column weights: the point's top 7 coordinates) and r1 (the rest) as LSB-first
// eq tables of (real, imag) pairs: open_and_verify's dfs over the reversed point
// halves (linearPC.cpp:693-731) with truepix::reverse_point applied first
void weights(const std::vector<u64>& pt, int lg_n, std::vector<u64>& r0, std::vector<u64>& r1)
{
    r0.assign(2 * kColumns, 0);
    r1.assign(2 * ((size_t)1 << (lg_n - 7)), 0);
    tp_eq_table_host(pt.data() + 2 * (lg_n - 7), 7, r0.data());
    tp_eq_table_host(pt.data(), lg_n - 7, r1.data());
}
// (real, imag) pairs -> the codeword's {img, real} order
std::vector<u64> swapped(const std::vector<u64>& v)
{
    std::vector<u64> o(v.size());
    for (size_t i = 0; i + 1 < v.size(); i += 2) {
        o[i] = v[i + 1];
        o[i + 1] = v[i];
    }
    return o;
}
u64 fsub(u64 a, u64 b) { return a >= b ? a - b : a + P61 - b; }

void write_result(bool ok, const u64 value[2])
{
    const char* path = getenv("TRUEPIX_ORION_RESULT_FILE");
    if (!path) return;
    FILE* f = fopen(path, "w");
    if (!f) {
        fprintf(stderr, "TruePix: cannot write %s\n", path);
        return;
    }
    fprintf(f, "{\n  \"ok\": %s,\n  \"value\": [%llu, %llu]\n}\n", ok ? "true" : "false",
            (unsigned long long)value[0], (unsigned long long)value[1]);
    fclose(f);
    printf("Wrote Orion opening result to %s\n", path);
}

bool nizk_mode()
{
    const char* m = getenv("TRUEPIX_ORION_MODE");
    return !(m && (!strcmp(m, "interactive") || !strcmp(m, "INTERACTIVE") || !strcmp(m, "interact")));
}

// ---- an opening (tensor_product_protocol, linearPC.cpp:426-662; Orion_zk :701-960) ----
// use_group1 1 and group -1: the plain opening; ZK: the masked polynomial over the
// even columns (use_group1 1, group 0) or the mask over the odd ones (0, 1).
// Writes `path`; returns the EC(y1) outcome (false also on errors). answer: (real, imag).
bool open_poly(const Layout& L, const Frame& F, const Poly& P, int use_group1, int group, const char* path,
               const std::vector<u64>& pt, u64 answer[2])
{
    const int qc = query_count();
    const long long msg_len = F.msg_len, cw_len = F.cw_len;
    if (group < 0)
        printf("Query count %d\nColumn size %d\nNumber of merkle pathes %d\nNumber of field elements %d\n", qc,
               kColumns, qc, qc * kColumns);
    std::vector<u64> r0, r1;
    weights(pt, L.lg_n, r0, r1);
    std::vector<long long> q(2 * (size_t)qc);   // the column queries, then the EC(y1) positions
    if (!lib_ok(tp_orion_open_queries2(P.root, (uint64_t)L.n, use_group1, r0.data(), kColumns, r1.data(), msg_len,
                                       cw_len, group, qc, q.data(), q.data() + qc), "opening transcript"))
        return false;
    Dev d_r0, d_r1, d_q, comb, ctree, ans, cols;
    if (!upload(d_r0, swapped(r0).data(), 8 * r0.size()) || !upload(d_r1, swapped(r1).data(), 8 * r1.size()) ||
        !upload(d_q, q.data(), 8 * q.size()) || !alloc(comb, 16 * (size_t)cw_len) ||
        !alloc(ctree, 64 * (size_t)F.leaves) || !alloc(ans, 16) || !alloc(cols, 16 * (size_t)qc * kColumns))
        return false;
    if (!lib_ok(tp_orion_combine_dev(P.rows.p, L.n, d_r0.p, comb.p, ctree.p, nullptr), "combine") ||
        !lib_ok(tp_orion_answer_dev(comb.p, msg_len, d_r1.p, ans.p, nullptr), "answer") ||
        !lib_ok(tp_orion_query_columns_dev(P.rows.p, L.n, d_q.p, qc, cols.p, nullptr), "queried columns"))
        return false;
    // the Merkle nodes of both trees at the queried leaves
    const int cap = qc * 64;
    std::vector<int> nodes(cap);
    const int nn = tp_orion_path_nodes(F.leaves, q.data(), qc, nodes.data(), cap);
    if (nn < 0) return lib_ok(-1, "Merkle paths");
    Dev d_nodes, com_dig, cmb_dig;
    if (!upload(d_nodes, nodes.data(), 4 * (size_t)nn) || !alloc(com_dig, 32 * (size_t)nn) ||
        !alloc(cmb_dig, 32 * (size_t)nn) ||
        !lib_ok(tp_orion_gather_nodes_dev(P.tree.p, 2 * F.leaves, d_nodes.p, nn, com_dig.p, nullptr), "Merkle nodes") ||
        !lib_ok(tp_orion_gather_nodes_dev(ctree.p, 2 * F.leaves, d_nodes.p, nn, cmb_dig.p, nullptr), "Merkle nodes"))
        return false;
    // EC(y1): the code of the combined message at the second batch of positions
    const double te = now();
    Dev enc;
    if (!alloc(enc, 16 * (size_t)cw_len) || !lib_ok(tp_orion_encode_dev(comb.p, msg_len, enc.p, nullptr), "EC(y1)"))
        return false;
    std::vector<u64> h_comb(2 * (size_t)cw_len), h_enc(2 * (size_t)cw_len), h_cols(2 * (size_t)qc * kColumns);
    std::vector<unsigned char> h_com(32 * (size_t)nn), h_cmb(32 * (size_t)nn), croot(32);
    u64 h_ans[2];
    if (!download(h_comb.data(), comb.p, 8 * h_comb.size()) || !download(h_enc.data(), enc.p, 8 * h_enc.size()) ||
        !download(h_cols.data(), cols.p, 8 * h_cols.size()) || !download(h_com.data(), com_dig.p, h_com.size()) ||
        !download(h_cmb.data(), cmb_dig.p, h_cmb.size()) ||
        !download(croot.data(), ctree.as<unsigned char>() + 32, 32) || !download(h_ans, ans.p, 16))
        return false;
    bool result = true;
    for (int i = qc; i < 2 * qc; ++i) {
        const size_t p = (size_t)q[i];
        if (h_enc[2 * p] != h_comb[2 * p] || h_enc[2 * p + 1] != h_comb[2 * p + 1]) result = false;
    }
    const double ec = now() - te;
    answer[0] = h_ans[1];
    answer[1] = h_ans[0];
    const long long proof_size = 32LL * 2 * nn + (long long)qc * kColumns * 16 + (long long)qc * 16;
    printf("EC(y1) code-switching time %lf\n", ec);
    printf("Proof size for tensor IOP %lld bytes\n", proof_size);
    printf("Proof size for P %lld bytes\n", proof_size);
    printf("Verification time %lf\n", ec);
    if (!result) return false;
    const long long size = tp_orion_opening_file_size(msg_len, cw_len, qc, nn, nn);
    std::vector<unsigned char> file((size_t)size);
    if (tp_orion_opening_file(L.n, msg_len, cw_len, h_ans, P.root, croot.data(), q.data(), qc, h_cols.data(),
                              h_comb.data(), nodes.data(), h_com.data(), nn, nodes.data(), h_cmb.data(), nn,
                              use_group1, file.data(), size) != size)
        return lib_ok(-1, "opening file");
    FILE* f = fopen(path, "wb");
    if (!f || fwrite(file.data(), 1, file.size(), f) != file.size()) {
        if (f) fclose(f);
        fprintf(stderr, "TruePix: failed to write NIZK proof %s\n", path);
        return false;
    }
    fclose(f);
    printf("ORION_NIZK_PROOF_BYTES %lld\nORION_NIZK_PROOF_FILE %s\n", size, path);
    return true;
}

// ---- an opening's checks (verify_opening_proof, linearPC.cpp:733-879; Orion_zk :1037-1200) ----
struct Reader {
    const std::vector<unsigned char>& b;
    size_t at = 0;
    bool ok = true;
    template <class T> T get()
    {
        T v{};
        if (at + sizeof(T) > b.size()) { ok = false; return v; }
        memcpy(&v, b.data() + at, sizeof(T));
        at += sizeof(T);
        return v;
    }
    const unsigned char* take(size_t n)
    {
        if (at + n > b.size()) { ok = false; return nullptr; }
        const unsigned char* p = b.data() + at;
        at += n;
        return p;
    }
};

// accepted?; answer (real, imag); vt: seconds of the checks
bool verify_poly(const Layout& L, const unsigned char* expected_root, int use_group1, int group, const char* path,
                 const std::vector<u64>& pt, u64 answer[2], double& vt)
{
    answer[0] = answer[1] = 0;
    std::vector<unsigned char> b;
    {
        std::ifstream f(path, std::ios::binary);
        if (!f) {
            fprintf(stderr, "TruePix: cannot read NIZK proof\n");
            return false;
        }
        b.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    }
    // OpeningProof::read_file (orion_proof.cpp:96-137)
    Reader R{b};
    const unsigned char* magic = R.take(8);
    const uint32_t version = R.get<uint32_t>(), group1 = R.get<uint32_t>();
    const u64 N = R.get<u64>(), csize = R.get<u64>(), msg_len = R.get<u64>(), cw_len = R.get<u64>();
    const uint32_t qc = R.get<uint32_t>();
    const unsigned char* ans = R.take(16);
    const unsigned char* com_root = R.take(32);
    const unsigned char* cmb_root = R.take(32);
    const bool sane = R.ok && !memcmp(magic, "ORIONPV1", 8) && version == 2 && msg_len <= (1ULL << 24) &&
                      cw_len <= (1ULL << 26) && qc <= (1u << 16);
    const unsigned char* col_q = sane ? R.take(8 * (size_t)qc) : nullptr;
    const unsigned char* cols = sane ? R.take(16 * (size_t)qc * kColumns) : nullptr;
    const unsigned char* combined = sane ? R.take(16 * (size_t)cw_len) : nullptr;
    const unsigned char* message = sane ? R.take(16 * (size_t)msg_len) : nullptr;
    std::vector<std::pair<uint32_t, const unsigned char*>> com, cmb;
    for (auto* list : {&com, &cmb}) {
        const u64 n = sane ? R.get<u64>() : 0;
        if (!R.ok || n > (1ULL << 24)) { R.ok = false; break; }
        for (u64 i = 0; i < n && R.ok; ++i) {
            const uint32_t idx = R.get<uint32_t>();
            const unsigned char* d = R.take(32);
            list->emplace_back(idx, d);
        }
    }
    if (!sane || !R.ok) {
        fprintf(stderr, "TruePix: cannot read NIZK proof\n");
        return false;
    }
    if (N != (u64)L.n || csize != kColumns || (TP_CLI_ZK && group1 != (uint32_t)use_group1)) {
        fprintf(stderr, "TruePix: proof layout mismatch\n");
        return false;
    }
    if (memcmp(com_root, expected_root, 32) != 0) {
        fprintf(stderr, "TruePix: proof com_root != expected\n");
        return false;
    }
    memcpy(answer, ans, 16);            // {img, real} in the file
    std::swap(answer[0], answer[1]);    // -> (real, imag)
    std::vector<u64> r0, r1;
    weights(pt, L.lg_n, r0, r1);
    std::vector<long long> q(2 * (size_t)qc);
    if (cw_len < 2 || msg_len != (u64)L.n / kColumns) {
        fprintf(stderr, "TruePix: proof layout mismatch\n");
        return false;
    }
    if (!lib_ok(tp_orion_open_queries2(com_root, N, use_group1, r0.data(), kColumns, r1.data(), (long long)msg_len,
                                       (long long)cw_len, group, (int)qc, q.data(), q.data() + qc),
                "opening transcript"))
        return false;
    for (uint32_t i = 0; i < qc; ++i) {
        long long got;
        memcpy(&got, col_q + 8 * i, 8);
        if (got != q[i]) {
            fprintf(stderr, "TruePix: FS column query mismatch at %u\n", i);
            return false;
        }
    }
    const double t0 = now();
    // sibling lists sorted by node index; the first entry of an index wins (as a map would)
    auto sorted = [](std::vector<std::pair<uint32_t, const unsigned char*>>& v, std::vector<uint32_t>& idx,
                     std::vector<unsigned char>& dig) {
        std::stable_sort(v.begin(), v.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        for (size_t i = 0; i < v.size(); ++i) {
            if (!idx.empty() && idx.back() == v[i].first) continue;
            idx.push_back(v[i].first);
            dig.insert(dig.end(), v[i].second, v[i].second + 32);
        }
    };
    std::vector<uint32_t> com_idx, cmb_idx;
    std::vector<unsigned char> com_dig, cmb_dig;
    sorted(com, com_idx, com_dig);
    sorted(cmb, cmb_idx, cmb_dig);
    if (qc == 0 || com_idx.empty() || cmb_idx.empty()) {
        fprintf(stderr, "TruePix: NIZK Merkle verify failed\n");
        return false;
    }
    Dev d_r0, d_q, d_cols, d_comb, d_msg, d_r1, d_ans, d_enc, d_ci, d_cd, d_bi, d_bd, d_flags;
    if (!upload(d_r0, swapped(r0).data(), 8 * r0.size()) || !upload(d_q, q.data(), 8 * q.size()) ||
        !upload(d_cols, cols, 16 * (size_t)qc * kColumns) || !upload(d_comb, combined, 16 * (size_t)cw_len) ||
        !upload(d_msg, message, 16 * (size_t)msg_len) || !upload(d_r1, swapped(r1).data(), 8 * r1.size()) ||
        !alloc(d_ans, 16) || !alloc(d_enc, 16 * (size_t)cw_len) ||
        !upload(d_ci, com_idx.data(), 4 * com_idx.size()) || !upload(d_cd, com_dig.data(), com_dig.size()) ||
        !upload(d_bi, cmb_idx.data(), 4 * cmb_idx.size()) || !upload(d_bd, cmb_dig.data(), cmb_dig.size()) ||
        !alloc(d_flags, 4 * (size_t)qc))
        return false;
    // the answer from the proof's combined message; EC(y1): its code at the second batch
    if (!lib_ok(tp_orion_answer_dev(d_msg.p, (long long)msg_len, d_r1.p, d_ans.p, nullptr), "answer") ||
        !lib_ok(tp_orion_encode_dev(d_msg.p, (long long)msg_len, d_enc.p, nullptr), "EC(y1)") ||
        !lib_ok(tp_orion_verify_opening_dev((long long)msg_len, (long long)cw_len, d_r0.p, d_q.p,
                                            d_q.as<long long>() + qc, (int)qc, d_cols.p, d_comb.p, d_enc.p, d_ci.p,
                                            d_cd.p, (int)com_idx.size(), d_bi.p, d_bd.p, (int)cmb_idx.size(),
                                            com_root, cmb_root, d_flags.as<int>(), nullptr),
                "opening checks"))
        return false;
    std::vector<int> flags(qc);
    u64 re_ans[2];
    if (!download(flags.data(), d_flags.p, 4 * (size_t)qc) || !download(re_ans, d_ans.p, 16)) return false;
    vt = now() - t0;
    // the reference's order: per query the column, then both paths; then the answer
    for (uint32_t i = 0; i < qc; ++i) {
        if (flags[i] & (1 | 16)) {
            fprintf(stderr, "TruePix: column linear combo mismatch\n");
            return false;
        }
        if (flags[i] & 6) {
            fprintf(stderr, "TruePix: NIZK Merkle verify failed\n");
            return false;
        }
    }
    if (re_ans[0] != answer[1] || re_ans[1] != answer[0]) {
        fprintf(stderr, "TruePix: answer recomputation mismatch\n");
        return false;
    }
    bool ec_ok = true;
    for (uint32_t i = 0; i < qc; ++i) ec_ok &= !(flags[i] & 8);
    if (!ec_ok) fprintf(stderr, "TruePix: EC(y1) code check failed\n");
    const long long proof_size =
        32LL * (long long)(com_idx.size() + cmb_idx.size()) + (long long)qc * kColumns * 16 + (long long)qc * 16;
    printf("EC(y1) code-switching time %lf\n", vt);
    printf("Proof size for tensor IOP %lld bytes\n", proof_size);
    printf("Verification time %lf\n", vt);
    return ec_ok;
}

bool device_ready()
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n < 1) {
        fprintf(stderr, "TruePix: no CUDA device: these programs run the commit and the opening on the GPU\n");
        return false;
    }
    return true;
}

bool root_matches(const Poly& P, const std::string& want, const char* label)
{
    const std::string got = root_hex(P.root);
    if (got == want) return true;
    if (label)
        fprintf(stderr, "TruePix: %s Merkle root mismatch\n  committed: %s\n  manifest:  %s\n", label, got.c_str(),
                want.c_str());
    else
        fprintf(stderr, "TruePix: Merkle root mismatch\n  committed: %s\n  manifest:  %s\n", got.c_str(), want.c_str());
    return false;
}

// ---- the phases -------------------------------------------------------------------
int run_commit(const Layout& lay)
{
    Input in;
    if (!load_input("input.txt", lay, in)) return 1;
    Frame F;
    if (TP_CLI_ZK) {
        u64 seed = 0;
        if (!mask_seed_create(seed) || !device_ready()) return 1;
        printf("Running fused mask commit...\n");
        const double t0 = now();
        if (!commit_frame_zk(lay, in, seed, F)) return 1;
        printf("Commit time(mask): %lf\n", now() - t0);
        return write_manifest(lay, root_hex(F.masked.root), root_hex(F.mask.root), true) ? 0 : 1;
    }
    if (!device_ready()) return 1;
    const double t0 = now();
    if (!commit_frame(lay, in, F)) return 1;
    printf("Commit time %lf\n", now() - t0);
    return write_manifest(lay, root_hex(F.plain.root), "", false) ? 0 : 1;
}

// manifest, input, (seed), point: the common front of prove and open
bool front(int phase, const Layout& lay, Manifest& man, Input& in, u64& seed, std::vector<u64>& pt)
{
    if (!read_manifest(man)) return false;
    if (TP_CLI_ZK && !man.zk) {
        fprintf(stderr, "TruePix: ZK Orion cannot open a non-ZK commitment\n");
        return false;
    }
    if (!TP_CLI_ZK && man.zk) {
        fprintf(stderr, "TruePix: non-ZK Orion cannot open a ZK commitment\n");
        return false;
    }
    if (!(lay == man.lay)) {
        fprintf(stderr, "TruePix: layout does not match the commit manifest\n");
        return false;
    }
    if (!load_input("input.txt", lay, in)) return false;
    if (TP_CLI_ZK && !mask_seed_read(seed)) return false;
    if (!load_point(lay.lg_n, pt)) {
        if (phase == 3) fprintf(stderr, "TruePix: refusing to open at a point unrelated to the GKR claim\n");
        return false;
    }
    if (!nizk_mode()) {
        fprintf(stderr, "TruePix: only the NIZK Orion mode is served (TRUEPIX_ORION_MODE=%s)\n",
                getenv("TRUEPIX_ORION_MODE"));
        return false;
    }
    return device_ready();
}

int run_prove(const Layout& lay)
{
    Manifest man;
    Input in;
    u64 seed = 0, mle[2] = {0, 0};
    std::vector<u64> pt;
    if (!front(2, lay, man, in, seed, pt)) return 1;
    Frame F;
    if (TP_CLI_ZK) {
        printf("Running fused mask commit...\n");
        const double t0 = now();
        if (!commit_frame_zk(lay, in, seed, F)) return 1;
        printf("Commit time(mask): %lf\n", now() - t0);
        if (!frame_mle(lay, in, F, pt, mle)) return 1;
        const bool root_masked = root_matches(F.masked, man.masked_root, "masked");
        u64 v_masked[2], v_mask[2];
        double t1 = now();
        const bool open_masked = open_poly(lay, F, F.masked, 1, 0, "orion_proof_masked.bin", pt, v_masked);
        printf("Open time(masked): %lf\nResult: %s\n", now() - t1, open_masked ? "succ" : "fail");
        const bool root_mask = root_matches(F.mask, man.mask_root, "mask");
        t1 = now();
        const bool open_mask = open_poly(lay, F, F.mask, 0, 1, "orion_proof_mask.bin", pt, v_mask);
        printf("Open time(mask): %lf\nResult: %s\n", now() - t1, open_mask ? "succ" : "fail");
        const bool consistent = fsub(v_masked[0], v_mask[0]) == mle[0] && fsub(v_masked[1], v_mask[1]) == mle[1];
        const bool ok = open_masked && open_mask && root_masked && root_mask && consistent;
        printf("TruePix prove: open_masked=%d open_mask=%d root_masked=%d root_mask=%d mle_consistent=%d -> ok=%d\n",
               (int)open_masked, (int)open_mask, (int)root_masked, (int)root_mask, (int)consistent, (int)ok);
        printf(ok ? "check pass\n" : "check notpass\n");
        return ok ? 0 : 1;
    }
    const double t0 = now();
    if (!commit_frame(lay, in, F)) return 1;
    printf("Commit time %lf\n", now() - t0);
    if (!frame_mle(lay, in, F, pt, mle)) return 1;
    const bool root_ok = root_matches(F.plain, man.masked_root, nullptr);
    const double t1 = now();
    u64 value[2] = {0, 0};
    const bool opened = open_poly(lay, F, F.plain, 1, -1, "orion_proof.bin", pt, value);
    printf("Open time %lf\n", now() - t1);
    printf("%s\n", opened ? "succ" : "fail");
    const bool consistent = value[0] == mle[0] && value[1] == mle[1];
    const bool ok = opened && root_ok && consistent;
    printf("TruePix prove: open=%d root=%d mle_consistent=%d -> ok=%d\n", (int)opened, (int)root_ok,
           (int)consistent, (int)ok);
    printf(ok ? "check pass\n" : "check notpass\n");
    return ok ? 0 : 1;
}

int run_open(const Layout& lay)
{
    Manifest man;
    Input in;
    u64 seed = 0, mle[2] = {0, 0}, value[2] = {0, 0};
    std::vector<u64> pt;
    if (!front(3, lay, man, in, seed, pt)) return 1;
    Frame F;   // the plaintext MLE only; nothing is committed here
    const double tm = now();
    if (!frame_mle(lay, in, F, pt, mle)) return 1;
    const double mle_seconds = now() - tm;
    bool ok;
    if (TP_CLI_ZK) {
        u64 v[2][2] = {{0, 0}, {0, 0}};
        bool opened[2] = {false, false}, root_ok[2] = {false, false};
        const char* labels[2] = {"masked", "mask"};
        const char* files[2] = {"orion_proof_masked.bin", "orion_proof_mask.bin"};
        const std::string* roots[2] = {&man.masked_root, &man.mask_root};
        for (int k = 0; k < 2; ++k) {
            printf(k == 0 ? "Running with mask...\n" : "Running without mask...\n");
            unsigned char expected[32];
            if (!root_from_hex(*roots[k], expected)) {
                fprintf(stderr, "TruePix: %s invalid root hex in manifest\n", labels[k]);
                continue;
            }
            root_ok[k] = true;
            double vt = 0;
            const double t1 = now();
            opened[k] = verify_poly(lay, expected, k == 0 ? 1 : 0, k, files[k], pt, v[k], vt);
            printf("Open time(%s): %lf\nResult: %s\n", labels[k], now() - t1, opened[k] ? "succ" : "fail");
        }
        value[0] = fsub(v[0][0], v[1][0]);
        value[1] = fsub(v[0][1], v[1][1]);
        const bool consistent = value[0] == mle[0] && value[1] == mle[1];
        if (!consistent)
            fprintf(stderr, "TruePix: verified opening %llu+%llui disagrees with the plaintext MLE %llu+%llui\n",
                    (unsigned long long)value[0], (unsigned long long)value[1], (unsigned long long)mle[0],
                    (unsigned long long)mle[1]);
        printf("MLE evaluation time %f\n", mle_seconds);
        ok = opened[0] && opened[1] && root_ok[0] && root_ok[1] && consistent;
        printf("TruePix open: children=1 open_masked=%d open_mask=%d root_masked=%d root_mask=%d mle_consistent=%d "
               "-> ok=%d\n", (int)opened[0], (int)opened[1], (int)root_ok[0], (int)root_ok[1], (int)consistent,
               (int)ok);
    } else {
        unsigned char expected[32];
        if (!root_from_hex(man.masked_root, expected)) {
            fprintf(stderr, "TruePix: invalid root hex in manifest\n");
            return 1;
        }
        const double t1 = now();
        double vt = 0;
        const bool opened = verify_poly(lay, expected, 1, -1, "orion_proof.bin", pt, value, vt);
        printf("Open time %lf\n", now() - t1);
        printf("%s\n", opened ? "succ" : "fail");
        const bool consistent = value[0] == mle[0] && value[1] == mle[1];
        if (!consistent)
            fprintf(stderr, "TruePix: verified opening %llu+%llui disagrees with the plaintext MLE %llu+%llui\n",
                    (unsigned long long)value[0], (unsigned long long)value[1], (unsigned long long)mle[0],
                    (unsigned long long)mle[1]);
        ok = opened && consistent;
        printf("TruePix open: open=%d root=%d mle_consistent=%d -> ok=%d\n", (int)opened, 1, (int)consistent,
               (int)ok);
    }
    printf(ok ? "check pass\n" : "check notpass\n");
    write_result(ok, value);
    return ok ? 0 : 1;
}

}  // namespace

int main(int argc, char** argv)
{
    int copies = 0, userandom = 0;
    if (!parse_args(argc, argv, copies, userandom)) return 1;
    const char* proto = getenv("TRUEPIX_PROTOCOL");
    if (!proto || !protocol_ok(proto)) {
        fprintf(stderr, "TruePix: only the TruePix protocol is served (set TRUEPIX_PROTOCOL=%s)\n", kProtocol);
        return 1;
    }
    if (userandom) {
        fprintf(stderr, "fp2-linked-v1 requires shared input.txt (userandom=0)\n");
        return 1;
    }
    Layout lay;
    if (!make_layout(copies, lay)) return 1;
    const int rc = TP_CLI_PHASE == 1 ? run_commit(lay) : TP_CLI_PHASE == 2 ? run_prove(lay) : run_open(lay);
    fflush(stdout);
    return rc;
}
