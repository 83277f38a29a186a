/*
 * ckks_b200.h - C ABI of the B200-native CKKS evaluation core.
 *
 * This is the drop-in boundary for the hot path of YI-HAIBO/cipher-pu (an
 * FPGA CKKS accelerator whose hot-path semantics live in its Python golden
 * models under scripts/ and tb/ref/).  Every entry point below names the
 * reference interface it replaces (path:line inside the reference project).
 *
 * Conventions
 *  - Plain C: no torch or CUDA types in signatures.  `stream` is a
 *    cudaStream_t passed as void* (NULL = legacy default stream).
 *  - All data pointers are DEVICE pointers owned by the caller; calls are
 *    stream-ordered and never synchronise the host.  The only allocating
 *    calls are ckks_ctx_create / ckks_ctx_destroy.
 *  - Polynomials are uint64 coefficient arrays, limb-major:
 *    [batch][poly][limb][N]; limb l of a call with prime_begin b uses the
 *    context prime b + l.  Values are canonical residues in [0, q).
 *  - Evaluation-domain ("NTT domain") arrays hold the evaluations in
 *    bit-reversed order (ckks_bitrev_permute converts to natural order).
 *  - Return value: 0 = ok, > 0 = invalid argument / unsupported, < 0 = CUDA
 *    error.  ckks_last_error() gives a message for the calling thread.
 */
#ifndef CKKS_B200_H
#define CKKS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ckks_ctx ckks_ctx;

enum {
  CKKS_OK = 0,
  CKKS_EINVAL = 1,
  CKKS_EUNSUPPORTED = 2,
  CKKS_ECUDA = -1,
  CKKS_ETIMEOUT = -2
};

/* ABI version (bumped on any signature change). */
int ckks_abi_version(void);

/* Message of the last failing call on this thread ("" if none). */
const char* ckks_last_error(void);

/*
 * Create a context: ring dimension N = 2^log_n (1 <= log_n <= 14) over
 * n_primes primes; the last n_special (0 or 1) are special (keyswitch)
 * primes.  psi[i] is a primitive 2N-th root of unity mod primes[i] or 0 when
 * 2N does not divide primes[i]-1 (negacyclic transforms are then refused for
 * that prime); omega[i] is a primitive N-th root (0 -> psi[i]^2).
 * Replaces the parameter path scripts/gen_modulus_chain.py:97 find_k_primes,
 * scripts/gen_omega_tables.py:85 derive_omega and :96 generate_table (the
 * twiddle ROM that rtl/m1/ntt_unit.sv:99-106 loads with $readmemh).
 * Allocates device memory (tables); the only allocating entry besides destroy.
 */
int ckks_ctx_create(int log_n, int n_primes, int n_special, const uint64_t* primes,
                    const uint64_t* psi, const uint64_t* omega, ckks_ctx** out);
int ckks_ctx_destroy(ckks_ctx* ctx);

/*
 * Launch-shape tuning of a context (used by the autotuner).  Parameters:
 *   CKKS_TUNE_CM_LOG_ELEMS: coefficients per thread of the ct-mult kernels
 *   as log2 (3 -> radix-8 passes with N/8 threads, 4 -> radix-16 with N/16;
 *   0 = default 3).
 *   CKKS_TUNE_CM_MIN_BLOCKS: CTAs per SM the ct-mult kernels' register
 *   budget targets (1 or 2; 2 is built for N = 2^12, 2^13 only; 0 = default).
 * The reference fixes its datapath shape at synthesis time
 * (rtl/m1/ntt_unit.sv:39-52 parameters).
 */
enum { CKKS_TUNE_CM_LOG_ELEMS = 0, CKKS_TUNE_CM_MIN_BLOCKS = 1 };
int ckks_ctx_set_tuning(ckks_ctx* ctx, int param, int value);

/*
 * In-place forward (inverse = 0) or inverse NTT of n_polys x n_limbs
 * polynomials, negacyclic (cyclic = 0, ring X^N + 1) or cyclic (X^N - 1).
 * Forward: natural coefficients -> bit-reversed evaluations; inverse: back,
 * including the N^-1 scale.
 * Replaces tb/ref/gen_ntt_reference.py:78 ntt / :111 intt,
 * scripts/gen_omega_tables.py:154 _ntt_dit / :188 _intt_dif and the
 * rtl/m1/ntt_unit.sv:53-75 start/done datapath.
 */
int ckks_ntt(const ckks_ctx* ctx, uint64_t* data, int n_polys, int prime_begin, int n_limbs,
             int inverse, int cyclic, void* stream);

/* out[row][i] = in[row][bitrev(i)] for n_rows rows of N words (out != in).
 * Converts between the bit-reversed evaluation order and the natural order
 * of tb/ref/gen_ntt_reference.py:78 ntt (natural-order output). */
int ckks_bitrev_permute(const ckks_ctx* ctx, uint64_t* out, const uint64_t* in, int n_rows,
                        void* stream);

/* out = a * b pointwise per limb (evaluation domain).
 * Replaces the S_MUL stage of rtl/m2/poly_mult.sv:221-234. */
int ckks_pointwise_mul(const ckks_ctx* ctx, uint64_t* out, const uint64_t* a, const uint64_t* b,
                       int n_polys, int prime_begin, int n_limbs, void* stream);

/* out = a +- b (mod q) elementwise over n words with one modulus q < 2^62.
 * Replaces scripts/verify_keyswitch.py:40 poly_add / :44 poly_sub. */
int ckks_vec_addsub(uint64_t* out, const uint64_t* a, const uint64_t* b, int64_t n, uint64_t q,
                    int subtract, void* stream);

/*
 * Polynomial product in the coefficient domain through NTT -> pointwise ->
 * INTT, fused in one kernel (one CTA per polynomial limb), negacyclic or
 * cyclic.  Replaces scripts/verify_keyswitch.py:48 poly_mult (negacyclic,
 * = scripts/verify_e2e_mult.py:56) and
 * tb/ref/gen_poly_mult_vectors_n12.py:103 poly_mult_via_ntt (cyclic), i.e.
 * the rtl/m2/poly_mult.sv NTT(A), NTT(B), S_MUL, INTT sequence.
 */
int ckks_poly_mul(const ckks_ctx* ctx, uint64_t* out, const uint64_t* a, const uint64_t* b,
                  int n_polys, int prime_begin, int n_limbs, int cyclic, void* stream);

/*
 * Exact product mod an arbitrary q < 2^45 that need not be NTT-friendly
 * (e.g. the toy q = 113 of scripts/gen_ntt_vectors.py:107-110): the integer
 * product is formed in the three-prime context `crt3` (primes > 2^44 each,
 * N = the same ring dimension), recombined by Garner CRT and reduced mod q.
 * Replaces scripts/verify_keyswitch.py:48 poly_mult for any modulus.
 */
int ckks_poly_mul_anyq(const ckks_ctx* crt3, uint64_t* out, const uint64_t* a, const uint64_t* b,
                       int n_polys, uint64_t q, int cyclic, void* stream);

/*
 * Single-pair relinearisation of the golden model, one prime:
 *   f0 = e0 + e2 * kb,  f1 = e1 - e2 * ka   (mod q, ring X^N + 1)
 * all inputs/outputs coefficient domain, n_polys independent instances.
 * Replaces scripts/verify_keyswitch.py:62 relin and rtl/m3/keyswitch_pipe.sv.
 */
int ckks_relin_single(const ckks_ctx* ctx, uint64_t* f0, uint64_t* f1, const uint64_t* e0,
                      const uint64_t* e1, const uint64_t* e2, const uint64_t* ka,
                      const uint64_t* kb, int n_polys, int prime, void* stream);

/*
 * Exact single-modulus rescale c' = round(c * q_out / q_in) mod q_out
 * (round half up), n words, q_in, q_out < 2^50.
 * Replaces scripts/verify_rescale.py:38 rescale_coeff / :56 rescale_poly.
 */
int ckks_rescale_exact(uint64_t* out, const uint64_t* in, int64_t n, uint64_t q_in,
                       uint64_t q_out, void* stream);

/*
 * Scaled rescale of the end-to-end golden:
 *   c' = floor((c * q_out + q_in / 2) / (q_in * 2^scale_bits)) mod q_out
 * Replaces scripts/verify_e2e_mult.py:70 rescale.
 */
int ckks_rescale_scaled(uint64_t* out, const uint64_t* in, int64_t n, uint64_t q_in,
                        uint64_t q_out, int scale_bits, void* stream);

/*
 * RNS rescale (drop the last limb with rounding): in [n_polys][level][N]
 * evaluation domain over q_0..q_{level-1} -> out [n_polys][level-1][N]:
 *   out_i = (x_i - [centred(x_{level-1})]_{q_i}) * q_{level-1}^-1  (mod q_i)
 * Replaces rtl/m5/rescale_rns.sv (CRT -> centre -> divide -> re-split) and
 * the rescale step of scripts/verify_e2e_mult.py:98-99 for an RNS basis.
 */
int ckks_rescale_rns(const ckks_ctx* ctx, uint64_t* out, const uint64_t* in, int n_polys,
                     int level, void* stream);

/*
 * Relinearisation key preparation: ksk [dnum = n_q][2][n_q + 1][N]
 * (evaluation domain, digit j, component k (0: b, 1: a), limb over
 * q_0..q_{n_q-1}, special) -> prepared [dnum][2][n_q + 1][N] pairs of
 * (value, Shoup quotient), i.e. 2x the words.  Context must have one special
 * prime.  Key generation itself is host-side (no reference counterpart:
 * the reference keyswitch key is one (a, b) pair, scripts/verify_keyswitch.py:151).
 */
int ckks_relin_key_prepare(const ckks_ctx* ctx, uint64_t* prepared, const uint64_t* ksk,
                           void* stream);

/* Scratch bytes needed by ckks_ct_mul_relin_rescale for (n_ct, level). */
size_t ckks_ct_mul_scratch_bytes(const ckks_ctx* ctx, int n_ct, int level);

/*
 * Batched homomorphic multiply: tensor product, hybrid relinearisation
 * keyswitch (dnum = level digits, one special prime: ModUp, key inner
 * product, ModDown) and RNS rescale, for n_ct independent pairs.
 *   ct_a, ct_b : [n_ct][2][level][N] evaluation domain over q_0..q_{level-1}
 *   key        : prepared relinearisation key (ckks_relin_key_prepare)
 *   out        : [n_ct][2][level-1][N] evaluation domain
 *   scratch    : caller-allocated device buffer of at least
 *                ckks_ct_mul_scratch_bytes(ctx, n_ct, level) bytes
 * Decryption convention m ~ c0 + c1 * s.
 * Replaces scripts/verify_e2e_mult.py:78 e2e_mult (tensor + relin +
 * rescale) and the controllers rtl/m4/e2e_ckks_mult_ctrl_m4.sv /
 * rtl/m5/e2e_rns_top.sv, generalised to an RNS basis with a hybrid key.
 */
int ckks_ct_mul_relin_rescale(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct_a,
                              const uint64_t* ct_b, const uint64_t* key, int n_ct, int level,
                              void* scratch, size_t scratch_bytes, void* stream);

/* Size of the static device scratch used by ckks_ct_mul_relin_rescale_noalloc. */
#define CKKS_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)

/*
 * ckks_ct_mul_relin_rescale without caller scratch and without any device
 * allocation.  No counterpart in the reference (an FPGA design has no device
 * allocator); added for callers that are handed only their input and output
 * buffers and cannot call cudaMalloc - a plugin inside a foreign runtime whose
 * host owns all device memory through its own pool, or a serving loop whose
 * pool has reserved the GPU so that a new allocation would fail or stall other
 * streams.  Same arguments and results as ckks_ct_mul_relin_rescale minus the
 * scratch pair; the caller still owns `out`, `ct_a`, `ct_b` and `key`.
 *  - Scratch comes from one static device array of CKKS_NOALLOC_SCRATCH_BYTES
 *    (32 MiB) that every GPU loading this library keeps until process exit.
 *    A call needing more (ckks_ct_mul_scratch_bytes(ctx, n_ct, level) > 32 MiB,
 *    i.e. more than 51 pairs at N = 2^12, L = 3) is rejected with
 *    CKKS_EINVAL and a message naming the largest accepted batch.
 *  - The first call on each device looks up the array's device address
 *    (cudaGetSymbolAddress, with that device current) and caches it; make
 *    that first call before any stream capture.
 *  - All calls on a device share the one array: calls whose executions
 *    overlap on the GPU (different streams, other host threads) race and
 *    corrupt each other's results.  Serialise them on one stream.
 *  - Nothing in the array needs clearing between calls (every word is written
 *    before it is read); it keeps the last call's intermediates.
 *  - Refused while the profiler below is enabled (it creates CUDA events).
 */
int ckks_ct_mul_relin_rescale_noalloc(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct_a,
                                      const uint64_t* ct_b, const uint64_t* key, int n_ct,
                                      int level, void* stream);

/*
 * Per-kernel device timing (tracing).  When enabled, the multi-kernel entry
 * points record CUDA events around each kernel on the launching stream;
 * ckks_profile_read(stage) resolves them and returns the accumulated device
 * milliseconds and launch count of a stage: 0 = ct-mult tensor, 1 = ct-mult
 * ModUp + key inner product, 2 = ct-mult ModDown + rescale, 3 = ckks_ntt.
 * The reference has no runtime tracing (its timing comes from Vivado reports
 * and the cycle model of scripts/exp_e17_energy_efficiency.py:36-65).
 */
int ckks_profile_enable(int on);
int ckks_profile_reset(void);
int ckks_profile_read(int stage, double* total_ms, long long* launches);

#ifdef __cplusplus
}
#endif

#endif /* CKKS_B200_H */
