// Parameter context: everything precomputed for one ring degree and modulus chain,
// resident in HBM for the lifetime of the context.
#pragma once

#include <cstdint>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "common.cuh"
#include "ntt.cuh"

namespace tb {

enum Scheme { SCHEME_RAW = 0, SCHEME_BFV = 1, SCHEME_CKKS = 2, SCHEME_BGV = 3 };

// Status codes returned through the C ABI (include/troy_b200.h).
enum Status {
    TB_OK = 0,
    TB_ERR_INVALID_ARGUMENT = 1,
    TB_ERR_UNSUPPORTED = 2,
    TB_ERR_CUDA = 3,
    TB_ERR_OUT_OF_MEMORY = 4,
    TB_ERR_NO_KEY = 5,
    TB_ERR_TIMEOUT = 6,
};

int status_from(cudaError_t e);
int set_error(int status, const std::string &msg);

// Offsets (in words) of the per-level RNS constants inside RnsLevel::d_consts.
// "pair" entries are Shoup operands stored as consecutive {operand, quotient}.
struct RnsOff {
    int q_mtip;        // pair[L]: m~ (Q/q_i)^-1 mod q_i
    int q_ip;          // pair[L]: (Q/q_i)^-1 mod q_i
    int M_qB;          // [bsk+1][L]: (Q/q_i) m~^-1 mod b_k (lift rows), last row (Q/q_i) mod m~
    int M_qB_fl;       // [bsk][L]: (Q/q_i) c_k mod b_k, c_k the floor constant of b_k
    int Qmt_b;         // pair[bsk]: Q m~^-1 mod b_k
    int tc_b;          // pair[bsk]: t c_k mod b_k
    int neg_inv_q_mt;  // 1: -Q^-1 mod m~
    int Qmod_b;        // pair[bsk]: Q mod b_k
    int inv_mt_b;      // pair[bsk]: m~^-1 mod b_k
    int t_q;           // pair[L]: t mod q_i
    int t_b;           // pair[bsk]: t mod b_k
    int inv_q_b;       // pair[bsk]: Q^-1 mod b_k
    int B_ip;          // pair[bB]: (P_B/B_k)^-1 mod B_k
    int tq_ip;         // pair[L]: t (Q/q_i)^-1 mod q_i
    int iqb_Bip;       // pair[bB]: Q^-1 (P_B/B_k)^-1 mod B_k (c_k of B_k; c of m_sk is Q^-1)
    int M_Bq;          // [L][bB]: (P_B/B_k) mod q_i
    int M_Bmsk;        // [bB]: (P_B/B_k) mod m_sk
    int inv_pb_msk;    // pair: P_B^-1 mod m_sk
    int pb_q;          // pair[L]: P_B mod q_i
    int negpb_q;       // pair[L]: q_i - (P_B mod q_i)
    int tg_q;          // pair[L]: t*gamma mod q_i
    int M_qtg;         // [2][L]: (Q/q_i) mod {t, gamma}
    int neg_inv_q_tg;  // [2]: -Q^-1 mod {t, gamma}
    int inv_gamma_t;   // 1: gamma^-1 mod t
    int M_qt;          // [L]: (Q/q_i) mod t
    int q_mod_t;       // 1: Q mod t
    int cdpt;          // pair[L]: floor(Q/t) mod q_i
    int plain_incr;    // [L]: (Q - t) mod q_i
    int total;
};

// RNS tool constants of one chain level (reference RNSTool::initialize,
// src/utils/rns.cpp:581-803, and the ContextData scalars of src/context.cpp:253-300),
// in the form the BEHZ / decrypt / plaintext-lift kernels use.
struct RnsLevel {
    int L = 0;                  // data limbs at this level (moduli chain[0..L-1])
    int bB = 0, bsk = 0;        // |B| and |Bsk| = |B| + 1
    uint64_t m_sk = 0, gamma = 0;
    RnsOff off{};
    uint64_t *d_consts = nullptr;
    Mod *d_bsk_mods = nullptr;  // Bsk = [B_0 .. B_{bB-1}, m_sk]
    int *d_bsk_idx = nullptr;   // table indices of the Bsk primes
    Mod gamma_mod{};            // Barrett ratio only
};

// Constants for dividing by the last prime of a chain prefix with rounding: for a
// prefix of Lfull primes (last = chain[Lfull-1]) and a kept prime q_j, j < Lfull-1.
// Key-switch mod-down uses Lfull = chain.size() (last = the special prime).
struct DropC {
    uint64_t inv, inv_quo;          // last^-1 mod q_j (Shoup)
    uint64_t fix;                   // q_j - ((last >> 1) mod q_j)
    uint64_t half_mod;              // (last >> 1) mod q_j
    uint64_t lastmod, lastmod_quo;  // last mod q_j (Shoup)
};

struct Context {
    int device = 0;
    int scheme = SCHEME_RAW;
    int logn = 0;
    uint32_t n = 0;
    std::vector<uint64_t> chain;      // key-level moduli, special prime last
    uint64_t t = 0;                   // plain modulus (0 for CKKS / raw)
    int plain_index = -1;             // table index of t when batching is possible
    std::vector<uint64_t> table_moduli;
    std::vector<Mod> h_mods;          // host copy (device table pointers inside)
    Mod *d_mods = nullptr;
    ulonglong2 *d_tables = nullptr;
    std::vector<RnsLevel> levels;     // levels[L] for L = 1 .. chain.size()
    DropC *d_drop = nullptr;          // [(Lfull) * K + j], K = chain.size()
    Mod t_mod{};                      // plain modulus (Barrett ratio only), value 0 for CKKS
    std::vector<uint64_t> inv_qlast_t;  // [Lfull]: chain[Lfull-1]^-1 mod t (BGV)
    // Galois NTT-domain permutation tables, built on first use per element.
    std::mutex galois_mu;
    std::unordered_map<uint32_t, uint32_t *> galois_ntt;
    uint32_t *d_slot_map = nullptr;   // batch-encoder slot -> coefficient map
    void *d_fft_roots = nullptr;      // CKKS special-FFT roots: [N] forward, [N] inverse (double2)
    uint64_t *noalloc_scratch = nullptr;  // device address of the static relinearize scratch on `device`
    ~Context();
};

int context_create(int scheme, uint64_t n, const uint64_t *moduli, int count, uint64_t t, Context **out);

// Launches the forward / inverse NTT over [polys][limbs][n] words; limb l uses table
// modulus first + l. lazy keeps outputs in [0, 4q) / [0, 2q).
int ntt_forward(const Context &c, const uint64_t *in, uint64_t *out, uint64_t polys, int first, int limbs,
                bool lazy, cudaStream_t s);
int ntt_inverse(const Context &c, const uint64_t *in, uint64_t *out, uint64_t polys, int first, int limbs,
                bool lazy, cudaStream_t s);

}  // namespace tb

// The opaque handle of the C ABI (include/troy_b200.h) around one parameter context.
struct tb_context {
    tb::Context *c;
};
