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
 *    stream-ordered and never synchronise the host.  Device memory is
 *    allocated only by ckks_ctx_create (tables), once per thread and
 *    device by ckks_sample_dgauss (its CDF table), once per context by the
 *    first ckks_ntt_tc call (its matrix images) and by ckks_batch_plan_create
 *    (the plan); every other entry uses caller buffers.
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
 * The parameter set as one plain struct (the C mirror of the Python
 * CkksParams): ring, primes (the last n_special special), optional roots
 * (NULL or 0 entries: derived as g^((q-1)/2N), resp. psi^2 or g^((q-1)/N),
 * with g the smallest generator of (Z/qZ)^*, exactly as the Python side
 * derives them), and the scheme constants a caller keeps with its keys
 * (scale Delta, error width sigma, sampler seed; the context stores them
 * and ckks_ctx_get_params returns them, the kernels do not read them).
 * ckks_ctx_create_params is ckks_ctx_create from such a struct.
 * ckks_ctx_get_params fills *out from a context; its pointers point into
 * the context and stay valid while it lives.
 * Replaces the parameter constants spread over scripts/gen_modulus_chain.py
 * (argparse, :229-238), the rtl/m1/ntt_unit.sv:39-52 module parameters and
 * the chain JSON rtl/m2/modulus_chain_chain4.json.
 */
typedef struct ckks_params {
  int32_t log_n;
  int32_t n_primes;
  int32_t n_special;
  int32_t reserved;  /* 0 */
  const uint64_t* primes;
  const uint64_t* psi;    /* NULL: derived */
  const uint64_t* omega;  /* NULL: derived */
  double scale;
  double sigma;
  uint64_t seed;
} ckks_params;
int ckks_ctx_create_params(const ckks_params* params, ckks_ctx** out);
int ckks_ctx_get_params(const ckks_ctx* ctx, ckks_params* out);

/*
 * Launch-shape tuning of a context (used by the autotuner).  Parameters:
 *   CKKS_TUNE_CM_LOG_ELEMS: coefficients per thread of the ct-mult and
 *   rotation kernels as log2 K (radix-2^K register passes with N / 2^K
 *   threads).  Built: K = 3, 4 for log N in [6, 14] (N / 8 <= 1024 threads
 *   for K = 3); K = 2 for log N in [10, 12]; K = 5 for log N in [10, 14],
 *   balanced budget only.  0 = default: 4 for N >= 2^10, else 3.
 *   CKKS_TUNE_CM_MIN_BLOCKS: register budget of the ct-mult kernels:
 *   1 = balanced (128 registers per thread, max(1, 512 / threads) CTAs per
 *   SM), 2 = tight (64 registers, twice the CTAs); 0 = default (balanced).
 *   CKKS_TUNE_CM_SPLIT: sub-batches of one ct-mult call, run on 4 internal
 *   streams (sub-batch h on stream h mod 4; 1..16; 0 = default: one per 64
 *   pairs, at most 4, from 128 pairs on, else 1).  The kernels of one
 *   sub-batch fill the partial last waves of the others (measured +12 % at
 *   256 pairs, N = 2^12, L = 3); 8 or 16 sub-batches of 32 or 16 pairs
 *   measured 8 % and 32 % slower there.
 *   CKKS_TUNE_CM_UNITS_PER_CTA: work units (limbs, target primes, output
 *   polynomials) each CTA of the ct-mult and rotation kernels processes in
 *   turn, 1..8 (0 = default 1: one CTA per unit); the grid shrinks by the
 *   same factor.
 *   CKKS_TUNE_CM_TENSOR_TMA: the ct-mult's first kernel (tensor product and
 *   INTT of d2): 1 = persistent, one CTA per resident slot, inputs staged in
 *   shared memory by bulk asynchronous copies (two stages of quarter limbs,
 *   mbarrier completion, bounded waits); 2 = one CTA per (pair, limb) with
 *   direct loads; 0 = default.
 *   CKKS_TUNE_CM_FUSED: ct-mult path.  0 = default = 2: the three kernels
 *   (tensor, ModUp + key inner product, ModDown + rescale) through scratch;
 *   1 = the fused kernel (one thread-block cluster of level + 1 CTAs per
 *   pair, intermediates exchanged through distributed shared memory and
 *   accumulated in TMEM, no scratch), built for log N in [10, 13] and level
 *   in [2, 7], refusing other shapes.  The fused kernel reads and writes only
 *   the compulsory bytes but measured 0.50-0.77x the three kernels' rate on
 *   B200 (its CTAs wait at cluster barriers), so it is not the default.
 *   ckks_ct_mul_scratch_bytes follows this choice (0 when fused).
 *   CKKS_TUNE_WAIT_CYCLES: limit, in SM cycles, of every bounded device-side
 *   wait of the context's kernels (a bulk copy landing in shared memory, a
 *   work-queue flag); on expiry a kernel records it for ckks_device_status,
 *   lets its own copies in flight land and returns.  0 = default
 *   (2^31 - 1 cycles, about 1.1 s at 1965 MHz).
 *   CKKS_TUNE_CM_MODUP_TMEM: where the three-kernel ct-mult's ModUp keeps
 *   its key inner-product accumulators: 1 = Tensor Memory (the CTA then
 *   needs only its transform buffer in shared memory and three 256-thread
 *   CTAs share an SM; built for radix 2^4 at N = 2^12, where it measured
 *   2.7-5.6 % faster), 2 = shared memory; 0 = default (TMEM where built).
 *   Results are identical.
 *   CKKS_TUNE_NTT_LOG_ELEMS: K of ckks_ntt, ckks_ct_mul_plain_rescale and
 *   ckks_mul_plain_multi, in [2, 5] for log N in [6, 14] with
 *   N / 2^K <= 1024 (0 = default: min(4, log N)).
 * The reference fixes its datapath shape at synthesis time
 * (rtl/m1/ntt_unit.sv:39-52 parameters).
 */
enum {
  CKKS_TUNE_CM_LOG_ELEMS = 0,
  CKKS_TUNE_CM_MIN_BLOCKS = 1,
  CKKS_TUNE_CM_SPLIT = 2,
  CKKS_TUNE_NTT_LOG_ELEMS = 3,
  CKKS_TUNE_CM_UNITS_PER_CTA = 4,
  CKKS_TUNE_CM_TENSOR_TMA = 5,
  CKKS_TUNE_WAIT_CYCLES = 6,
  CKKS_TUNE_CM_FUSED = 7,
  CKKS_TUNE_CM_MODUP_TMEM = 8
};
int ckks_ctx_set_tuning(ckks_ctx* ctx, int param, int value);

/*
 * Device-side status of the kernels that wait with a bounded spin (the
 * TMA-fed ct-mult tensor kernel on its copies, the tensor-core linear
 * layer and transform on their MMA completions, the persistent batch kernel on its work
 * queue's dependency counters): CKKS_ETIMEOUT (and the
 * count in ckks_last_error) when any such wait on the current device expired
 * since the last call, which leaves those outputs incomplete; CKKS_OK
 * otherwise.  Synchronises the device; clears the count.
 */
int ckks_device_status(void);

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

/*
 * The forward negacyclic NTT of ckks_ntt (same layout, output order and
 * results) computed on the tensor cores: N = 2^12 as a 64 x 64 four-step
 * transform whose two 64-point stages are int8 byte-limb matrix products
 * (tcgen05.mma kind::i8), exact through an FP64 recombination.  N = 2^12
 * contexts only; the first call builds the context's matrix images (about
 * 112 KB per prime, device memory freed with the context) and should come
 * before any stream capture.  The engine the task statement conditions
 * tensor-core use on; ckks_ntt stays the default (it is faster).
 * Replaces tb/ref/gen_ntt_reference.py:78 ntt (forward, with the
 * negacyclic twist), like ckks_ntt.
 */
int ckks_ntt_tc(ckks_ctx* ctx, uint64_t* data, int n_polys, int prime_begin, int n_limbs, void* stream);

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
 * q_0..q_{n_q-1}, special) -> prepared [dnum][2][n_q + 1] blocks of 2N
 * doubles: the N key values w (exact) followed by their N correctly rounded
 * quotients w / q (the operands of the FP64 modular product), i.e. 2x the
 * words.  Context must have one special
 * prime.  Key generation itself is host-side (no reference counterpart:
 * the reference keyswitch key is one (a, b) pair, scripts/verify_keyswitch.py:151).
 */
int ckks_relin_key_prepare(const ckks_ctx* ctx, uint64_t* prepared, const uint64_t* ksk,
                           void* stream);

/* Scratch bytes needed by ckks_ct_mul_relin_rescale for (n_ct, level): 0
 * when the call takes the fused kernel (see CKKS_TUNE_CM_FUSED), else the
 * three-kernel path's (6 level + 2) limbs per pair. */
size_t ckks_ct_mul_scratch_bytes(const ckks_ctx* ctx, int n_ct, int level);

/*
 * Batched homomorphic multiply: tensor product, hybrid relinearisation
 * keyswitch (dnum = level digits, one special prime: ModUp, key inner
 * product, ModDown) and RNS rescale, for n_ct independent pairs.
 *   ct_a, ct_b : [n_ct][2][level][N] evaluation domain over q_0..q_{level-1}
 *   key        : prepared relinearisation key (ckks_relin_key_prepare)
 *   out        : [n_ct][2][level-1][N] evaluation domain
 *   scratch    : caller-allocated device buffer of at least
 *                ckks_ct_mul_scratch_bytes(ctx, n_ct, level) bytes (may be
 *                NULL when that is 0: the fused kernel needs none)
 * Decryption convention m ~ c0 + c1 * s.
 * Replaces scripts/verify_e2e_mult.py:78 e2e_mult (tensor + relin +
 * rescale) and the controllers rtl/m4/e2e_ckks_mult_ctrl_m4.sv /
 * rtl/m5/e2e_rns_top.sv, generalised to an RNS basis with a hybrid key.
 */
int ckks_ct_mul_relin_rescale(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct_a,
                              const uint64_t* ct_b, const uint64_t* key, int n_ct, int level,
                              void* scratch, size_t scratch_bytes, void* stream);

/*
 * ckks_ct_mul_relin_rescale on HOST buffers: out_host, a_host, b_host are
 * host arrays in the same layouts ([n_ct][2][level][N] in, [n_ct][2][level-1][N]
 * out); `key` is the prepared key in device memory.  The batch is cut into
 * chunks of `chunk` pairs pipelined over three internal streams (host->device
 * copy, kernels and device->host copy of consecutive chunks overlap).  The
 * device workspace (caller-owned) must hold
 * ckks_ct_mul_host_workspace_bytes(ctx, chunk, level) bytes.  Work already
 * queued on `stream` is ordered before the call; the call returns when all
 * outputs are in host memory.  Host buffers should be page-locked for the
 * copies to overlap.  Replaces the host side of scripts/verify_e2e_mult.py:78
 * e2e_mult (list[int] in, list[int] out) for batches.
 */
size_t ckks_ct_mul_host_workspace_bytes(const ckks_ctx* ctx, int chunk, int level);
int ckks_ct_mul_relin_rescale_host(const ckks_ctx* ctx, uint64_t* out_host, const uint64_t* a_host,
                                   const uint64_t* b_host, const uint64_t* key, int n_ct, int level,
                                   int chunk, void* workspace, size_t workspace_bytes,
                                   void* stream);

/*
 * CKKS slot encoding (FP64 canonical embedding, scale Delta):
 * slots [n_polys][n_slots] complex doubles (re, im interleaved), n_slots <=
 * N/2; slot k is the evaluation at Phi^(2k+1), Phi = exp(i pi / N), with its
 * conjugate at N-1-k; coefficients round(Delta * m) -> out [n_polys][level][N]
 * in the evaluation domain.  Replaces scripts/verify_multi_slot_simd.py:75
 * encode (and :42 neg_ifft) at production N (log_n <= 13).
 */
int ckks_encode(const ckks_ctx* ctx, uint64_t* out, const double* slots, int n_polys, int n_slots,
                int level, double scale, void* stream);

/*
 * Decoding: in [n_polys][level][N] COEFFICIENT-domain residues (e.g. the
 * output of ckks_decrypt) -> balanced CRT to the centred integer -> / scale ->
 * slots [n_polys][n_slots] complex.  Replaces scripts/verify_multi_slot_simd.py:88
 * decode (and :32 neg_fft).
 */
int ckks_decode(const ckks_ctx* ctx, double* slots, const uint64_t* in_coef, int n_polys,
                int n_slots, int level, double scale, void* stream);

/*
 * Decryption: ct [n_ct][2][level][N] (evaluation domain) -> out
 * [n_ct][level][N] coefficient-domain residues of c0 + c1 s.  s_eval: the
 * secret in the evaluation domain, [n_primes][N] over all context primes.
 * Replaces scripts/exp_e11_ckks_e2e_real.py:90 rlwe_decrypt and
 * scripts/exp_e24_rotation_bootstrap.py:126 decrypt_exact_int (their
 * (b, a) with b = a s + e + m equals (c0, c1) = (b, -a) here).
 */
int ckks_decrypt(const ckks_ctx* ctx, uint64_t* out_coef, const uint64_t* ct,
                 const uint64_t* s_eval, int n_ct, int level, void* stream);

/*
 * Encryption under the secret: c1 = a, c0 = -a s + NTT(e) + m over
 * q_0..q_{level-1}.  m_eval [n_ct][level][N] plaintext (evaluation domain, or
 * NULL for zero), a [n_ct][level][N] uniform residues, e [n_ct][N] small
 * signed errors.  Host samplers provide a and e (seeded).  Replaces
 * scripts/exp_e11_ckks_e2e_real.py:72 rlwe_encrypt and
 * scripts/exp_e24_rotation_bootstrap.py:209 rlwe_encrypt_mint.
 */
int ckks_encrypt(const ckks_ctx* ctx, uint64_t* out, const uint64_t* m_eval,
                 const uint64_t* s_eval, const uint64_t* a, const int64_t* e, int n_ct, int level,
                 void* stream);

/*
 * DARE refresh (decrypt -> re-encrypt): the centred integer m_int + e_old of
 * each ciphertext at level_in (balanced CRT over its limbs) is divided by
 * 2^shift_bits with rounding (0 keeps the scale) and encrypted afresh with a,
 * e at level_out (which may exceed level_in: the modulus is restored).
 * ct [n_ct][2][level_in][N] -> out [n_ct][2][level_out][N];
 * a [n_ct][level_out][N]; e [n_ct][N]; scratch >= ckks_dare_scratch_bytes.
 * With shift_bits > 0 the integer must satisfy |x| < 2^127.
 * Replaces scripts/exp_e24_rotation_bootstrap.py:287 reencrypt.
 */
size_t ckks_dare_scratch_bytes(const ckks_ctx* ctx, int n_ct, int level_in);
int ckks_dare_refresh(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct, const uint64_t* s_eval,
                      const uint64_t* a_fresh, const int64_t* e_fresh, int n_ct, int level_in,
                      int level_out, int shift_bits, void* scratch, size_t scratch_bytes,
                      void* stream);

/*
 * Noise monitor: per row of row_len residues mod q, the exact sum of
 * min(c, q - c)^2 as a 128-bit integer out_sum[2*row] (low) / [2*row+1]
 * (high); E = sum / row_len.  Replaces rtl/m4/noise_monitor.sv:42-129 and
 * scripts/verify_m4_h_multilayer.py:162 noise_monitor_energy.
 */
int ckks_noise_energy(uint64_t* out_sum, const uint64_t* in, int n_rows, int row_len, uint64_t q,
                      void* stream);

/*
 * The noise monitor with its accumulator width and saturation flag: as
 * ckks_noise_energy, plus saturated[row] = 1 when the exact sum reaches
 * 2^acc_bits (1 <= acc_bits <= 128), in which case the reported sum is
 * 2^acc_bits - 1.  acc_bits = 106 is the RTL's ACC_W.  The flag marks a
 * window whose noise left the monitor's range - a corrupted ciphertext or
 * key, or a decryption that wrapped around q.  Replaces the `saturated`
 * output of rtl/m4/noise_monitor.sv:30,62-73.
 */
int ckks_noise_energy_sat(uint64_t* out_sum, uint8_t* saturated, const uint64_t* in, int n_rows,
                          int row_len, uint64_t q, int acc_bits, void* stream);

/*
 * Slot SNR sums: per row, out[2*row] = sum |ref|^2, out[2*row+1] =
 * sum |dec - ref|^2 over row_len values (complex when complex_vals != 0).
 * SNR_dB = 10 log10(out0 / out1).  The decrypt-based SNR probe of the gear
 * loop (the reference estimates r_hat from decrypted vs plaintext values,
 * scripts/exp_e11_ckks_e2e_real.py:169 estimate_r_hat).
 */
int ckks_snr_sums(double* out, const double* dec, const double* ref, int n_rows, int row_len,
                  int complex_vals, void* stream);

/*
 * Block sparsity of a weight array: flat blocks of `block` weights whose
 * max |w| < threshold are zeroed; keep[b] (may be NULL) = 1 for kept blocks.
 * Replaces scripts/exp_e10_sparsity_sweep_v2.py:102 apply_block_sparse_mask
 * and rtl/m4/block_sparse_mask.sv.
 */
int ckks_block_sparse_mask(double* out, uint8_t* keep, const double* w, int64_t n, int block,
                           double threshold, void* stream);

/*
 * Output block skip of the approximate multiplier: per row, blocks of
 * `block` residues with max min(x, q - x) < threshold are zeroed when
 * use_approx and threshold != 0; skipped[row] = number of zeroed blocks.
 * Replaces scripts/verify_m4_d_approx_mult.py:50 post_process_block and
 * rtl/m4/approx_poly_mult.sv:1-44 (block mode).
 */
int ckks_block_post_process(uint64_t* out, int32_t* skipped, const uint64_t* in, int n_rows,
                            int row_len, int block, uint64_t q, uint64_t threshold, int use_approx,
                            void* stream);

/*
 * RNS split / merge over up to 8 primes (< 2^62, given in host memory).
 * split: in [n][words] little-endian integers (two's complement when
 *        centered) -> out [n_primes][n] residues.
 * merge: in [n_primes][n] residues -> out [n][words] integers via Garner CRT,
 *        in [0, M) or, when centered, the representative in (-M/2, M/2]
 *        (two's complement).
 * Replace rtl/m5/rns_split.sv:58-62 and rtl/m5/rns_merge.sv:84-135
 * (p1/p2/p3 = 77309411329, 206158430209, 2061584302081; M 115 bits).
 */
int ckks_rns_split(const uint64_t* primes, int n_primes, uint64_t* out, const uint64_t* in,
                   int64_t n, int words, int centered, void* stream);
int ckks_rns_merge(const uint64_t* primes, int n_primes, uint64_t* out, const uint64_t* in,
                   int64_t n, int words, int centered, void* stream);

/*
 * Energy-threshold gear controller (host state machine, no device work):
 * energy >= thresh[0] -> gear 0, >= thresh[1] -> 1, >= thresh[2] -> 2, else 3;
 * with hysteresis an upgrade (higher gear) takes effect after hyst_cnt
 * agreeing candidates while a downgrade is immediate; manual override.
 * Reset state: gear 3.  Replaces rtl/m4/adaptive_gear_ctrl.sv:43-99.
 */
typedef struct ckks_gear_ctrl {
  uint64_t thresh_lo[3], thresh_hi[3];
  int hyst_cnt, gear, counter, candidate;
} ckks_gear_ctrl;
int ckks_gear_ctrl_init(ckks_gear_ctrl* g, const uint64_t thresh_lo[3], const uint64_t thresh_hi[3],
                        int hyst_cnt);
int ckks_gear_ctrl_raw(const ckks_gear_ctrl* g, uint64_t energy_lo, uint64_t energy_hi);
int ckks_gear_ctrl_flush(ckks_gear_ctrl* g, uint64_t energy_lo, uint64_t energy_hi,
                         int hysteresis_en, int manual_en, int manual_gear);

/*
 * Seeded counter-based sampling (Philox4x32-10): element i of stream
 * `stream_id` depends only on (seed, stream_id, i).
 *  uniform: out [n_polys][n_limbs][N] residues uniform mod the limb primes;
 *  ternary: out[n] in {-1, 0, 1} uniform (the secret distribution);
 *  dgauss:  out[n] discrete Gaussian of width sigma (<= 16), tail cut at
 *           12 sigma (allocates a small CDF table once per thread and device).
 * The reference samples with numpy / random (scripts/exp_e33_real_ciphertext.py:75
 * dgauss, :153 ternary; scripts/exp_e11_ckks_e2e_real.py:72 uniform a).
 */
int ckks_sample_uniform(const ckks_ctx* ctx, uint64_t* out, int n_polys, int prime_begin,
                        int n_limbs, uint64_t seed, uint64_t stream_id, void* stream);
int ckks_sample_ternary(int64_t* out, int64_t n, uint64_t seed, uint64_t stream_id, void* stream);
int ckks_sample_dgauss(int64_t* out, int64_t n, double sigma, uint64_t seed, uint64_t stream_id,
                       void* stream);

/*
 * Encrypted linear layer with plaintext integer weights and 4x4 block
 * sparsity: out[o] = sum_f w[o][f] * in[f] (+ bias[o] on component 0), exact
 * mod every limb prime (< 2^47).  in [n_in][2][level][N], out
 * [n_out][2][level][N] (evaluation domain); w int32 [n_out][n_in] with
 * |w| < 2^24; bias int64 [n_out] or NULL; block_keep uint8
 * [ceil(n_out/4)][ceil(n_in/4)] (1 = compute the 4x4 block) or NULL = dense;
 * n_in <= 2048.  Zero blocks are skipped, so the work scales with the kept
 * fraction.  Replaces the encrypted FC layer of
 * scripts/exp_e11_ckks_e2e_real.py:142 encrypted_linear_layer and
 * rtl/m4/fc_layer_e2e.sv with slot-packed (SIMD over samples) ciphertexts.
 */
int ckks_linear_plain_weights(const ckks_ctx* ctx, uint64_t* out, const uint64_t* in,
                              const int32_t* w, const int64_t* bias, const uint8_t* block_keep,
                              int n_out, int n_in, int level, void* stream);

/*
 * The same encrypted linear layer on the tensor cores (tcgen05.mma kind::i8,
 * accumulators in TMEM): residues split into 6 unsigned bytes, weights into 3
 * balanced signed bytes, the 18 byte GEMMs accumulated exactly in int32 per
 * limb sum and recombined mod q in the epilogue.  Bit-identical to
 * ckks_linear_plain_weights.  Weights first go through ckks_linear_tc_pack
 * (host memory in and out, once per weight matrix and block mask; |w| <=
 * 8355711 = 127 (1 + 256 + 256^2), else CKKS_EINVAL), and the packed buffer
 * (ckks_linear_tc_packed_bytes, copied to the device, 16-byte aligned) is
 * passed here.  The 4x4 block mask is applied by the pack; dropped blocks are
 * multiplied as zeros (the tensor-core work does not shrink with sparsity).
 * n_in <= 2048, N >= 32.  Replaces the same reference layer as
 * ckks_linear_plain_weights (scripts/exp_e11_ckks_e2e_real.py:142).
 */
size_t ckks_linear_tc_packed_bytes(int n_out, int n_in);
int ckks_linear_tc_pack(void* packed_host, size_t packed_bytes, const int32_t* w_host,
                        const uint8_t* block_keep_host, int n_out, int n_in);
int ckks_linear_plain_weights_tc(const ckks_ctx* ctx, uint64_t* out, const uint64_t* in,
                                 const void* packed, const int64_t* bias, int n_out, int n_in,
                                 int level, void* stream);

/*
 * Learned gear controller network (no counterpart in the reference, whose
 * gear logic is thresholds + hysteresis, rtl/m4/adaptive_gear_ctrl.sv): a
 * 16 -> 64 -> 64 -> 4 FP32 MLP with ReLU hidden layers predicting the
 * post-layer SNR of each gear.  params: ckks_gear_mlp_param_count() floats
 * laid out W1[64][16], b1[64], W2[64][64], b2[64], W3[4][64], b3[4].
 *  forward:  x [batch][16] -> y [batch][4]; cache [batch][128] (hidden
 *            activations, needed by backward) may be NULL.
 *  backward: loss = (1/batch) sum mask * (y - target)^2 (mask may be NULL);
 *            grad [param_count]; dcache scratch [batch][132]; deterministic.
 *  adam:     in-place Adam step (bias-corrected, step counts from 1).
 */
int ckks_gear_mlp_param_count(void);
int ckks_gear_mlp_forward(const float* params, const float* x, float* y, float* cache, int batch,
                          void* stream);
int ckks_gear_mlp_backward(const float* params, const float* x, const float* cache, const float* y,
                           const float* target, const float* mask, float* grad, float* dcache,
                           int batch, void* stream);
int ckks_gear_mlp_adam(float* params, const float* grad, float* m, float* v, int step, float lr,
                       float beta1, float beta2, float eps, void* stream);

/*
 * Ciphertext x plaintext multiply fused with the RNS rescale:
 * ct [n_ct][2][level][N], pt [level][N] shared (pt_per_ct = 0) or
 * [n_ct][level][N] (pt_per_ct = 1), all evaluation domain ->
 * out [n_ct][2][level-1][N].  Replaces scripts/exp_e11_ckks_e2e_real.py:102
 * rlwe_mul_plain (and scripts/exp_e24_rotation_bootstrap.py mul_plain_exact)
 * followed by the rescale of rtl/m5/rescale_rns.sv.
 */
int ckks_ct_mul_plain_rescale(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct,
                              const uint64_t* pt, int pt_per_ct, int n_ct, int level, void* stream);

/*
 * Modular-multiply throughput microbenchmark (compute roofline of the
 * NTT-bound kernels): n_blocks x threads threads each run 8 independent
 * chains of `iters` lazy modular multiplies by w mod q (q < 2^47) - kind 0:
 * integer Shoup, 1: FP64 double-word, 2: both interleaved.  out receives one
 * word per thread (to keep the work alive).  Time it with events on `stream`:
 * modmul/s = n_blocks * threads * iters * 8 / seconds.
 */
int ckks_modmul_peak(uint64_t* out, int n_blocks, int threads, int iters, int kind, uint64_t q,
                     uint64_t w, void* stream);

/*
 * Ring automorphism psi_nu(f)(X) = f(X^nu) mod (X^N + 1) of n_polys x n_limbs
 * limbs (primes prime_begin ..), out != in.  Coefficient domain
 * (eval_domain = 0): any nu >= 0 (coefficient k goes to nu k mod N with sign
 * (-1)^floor(nu k / N), colliding terms summed), the reference's
 * scripts/exp_e24_rotation_bootstrap.py:143 automorphism_exact and :167
 * automorphism_key_exact.  Evaluation domain (eval_domain = 1, bit-reversed
 * order of ckks_ntt, negacyclic primes): odd nu, a permutation of the slots.
 */
int ckks_automorphism(const ckks_ctx* ctx, uint64_t* out, const uint64_t* in, int n_polys,
                      int prime_begin, int n_limbs, uint64_t nu, int eval_domain, void* stream);

/*
 * Coefficient-domain product with the monomial X^nu in Z_q[X]/(X^N + 1)
 * (nu taken mod 2N; X^N = -1), out != in.  Replaces
 * scripts/exp_e24_rotation_bootstrap.py:189 poly_mul_x_power and :232 rotate
 * (ct x X^nu), which agree with it for nu < N (they reduce nu mod N first).
 */
int ckks_mul_monomial(const ckks_ctx* ctx, uint64_t* out, const uint64_t* in, int n_polys,
                      int prime_begin, int n_limbs, uint64_t nu, void* stream);

/*
 * Coefficient-encoded inner products (the Conv + GAP fusion): every
 * ciphertext (b, a) of ct [n_ct][2][N] (coefficient domain, residues mod
 * primes[prime]) times every plaintext polynomial of w_hat [n_w][N], given in
 * the evaluation domain (negacyclic forward ckks_ntt of the scattered weight
 * polynomials, once per model) -> out [n_ct][n_w][2][N], coefficient domain,
 * canonical.  One NTT per ciphertext polynomial, one INTT per filter.
 * Replaces scripts/exp_e24_rotation_bootstrap.py:136 mul_plain_exact as
 * :615 encrypted_inference_fused calls it once per filter (through :263
 * inner_product, whose weights :241 scatter_w places).
 */
int ckks_mul_plain_multi(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct, const uint64_t* w_hat,
                         int n_ct, int n_w, int prime, void* stream);

/*
 * Constant coefficient of the decryption (b - a s) mod q of each ciphertext
 * of ct [n_ct][2][N] (coefficient domain), centred to (-q/2, q/2] (q odd),
 * with s the N residues of the secret key mod q = primes[prime]; the a and s
 * words must be below 2^52 (residues in [0, q) are).  Replaces
 * dec[0] of scripts/exp_e24_rotation_bootstrap.py:109 decrypt_exact, the one
 * coefficient :263 inner_product and :278 coef_sum read.
 */
int ckks_decrypt_coef0(const ckks_ctx* ctx, int64_t* out, const uint64_t* ct, const uint64_t* s,
                       long long n_ct, int prime, void* stream);

/*
 * Homomorphic automorphism with key switching ("rotation"): ct [n_ct][2][level][N]
 * (evaluation domain) -> out [n_ct][2][level][N] decrypting to psi_nu(m) under
 * the same secret, nu odd.  `key` is a Galois key prepared by
 * ckks_relin_key_prepare from ksk[j] = (-a_j s + e_j + delta_ij (P mod q_j)
 * psi_nu(s), a_j) over the L + 1 primes (the relinearisation key with s^2
 * replaced by psi_nu(s)); hybrid key switching with dnum = level digits, no
 * rescale.  Scratch: ckks_rotate_scratch_bytes(ctx, n_ct, level) bytes.
 * The reference rotates coefficient-encoded messages by X^nu without key
 * switching (scripts/exp_e24_rotation_bootstrap.py:232 rotate); slot
 * rotations of slot-packed ciphertexts need this Galois form.
 */
size_t ckks_rotate_scratch_bytes(const ckks_ctx* ctx, int n_ct, int level);
int ckks_rotate(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct, const uint64_t* key, int n_ct,
                int level, uint64_t nu, void* scratch, size_t scratch_bytes, void* stream);

/*
 * First-order masked single-pair relinearisation: like ckks_relin_single with
 * the key given as two additive shares a = a1 + a2, b = b1 + b2 (mod q), each
 * share processed on its own and only the products combined:
 * f0 = e0 + e2 b1 + e2 b2, f1 = e1 - e2 a1 - e2 a2 (coefficient domain, one
 * NTT-friendly prime).  Results equal ckks_relin_single's with (a, b).
 * Replaces rtl/m3/keyswitch_pipe_masked.sv:1-27 (two-pass arithmetic masking).
 */
int ckks_relin_single_masked(const ckks_ctx* ctx, uint64_t* f0, uint64_t* f1, const uint64_t* e0,
                             const uint64_t* e1, const uint64_t* e2, const uint64_t* a1,
                             const uint64_t* b1, const uint64_t* a2, const uint64_t* b2, int n_polys,
                             int prime, void* stream);

/*
 * Elementwise ciphertext arithmetic over ct [n_ct][2][level][N] (any domain,
 * limbs over q_0 .. q_{level-1}): out = a + b or a - b (subtract != 0);
 * out = m in (ct x integer constant, every limb times m mod q_i: the scale
 * is multiplied by m); out = in + c on component 0, c given by its residues
 * c_res[l] = c mod q_l (host array of `level` words; c may exceed 64 bits):
 * adds c to the plaintext's every slot in the evaluation domain / to its
 * constant coefficient in the coefficient domain.  In-place calls (out ==
 * input) are allowed.
 * The reference adds polynomials with scripts/verify_keyswitch.py:40
 * poly_add / :44 poly_sub and scales by integer weights in
 * scripts/exp_e11_ckks_e2e_real.py:102 rlwe_mul_plain.
 */
int ckks_ct_add(const ckks_ctx* ctx, uint64_t* out, const uint64_t* a, const uint64_t* b, int n_ct,
                int level, int subtract, void* stream);
int ckks_ct_mul_const(const ckks_ctx* ctx, uint64_t* out, const uint64_t* in, int n_ct, int level,
                      int64_t m, void* stream);
int ckks_ct_add_const(const ckks_ctx* ctx, uint64_t* out, const uint64_t* in, int n_ct, int level,
                      const uint64_t* c_res, void* stream);

/*
 * 48-bit wire format of residues (< 2^47): each word as its 6 low bytes,
 * little-endian, densely packed (n words <-> 6 n bytes), device to device;
 * both buffers 16-byte aligned.  Bits above 47 are not carried.
 */
int ckks_unpack48(uint64_t* out, const void* in, long long n, void* stream);
int ckks_pack48(void* out, const uint64_t* in, long long n, void* stream);

/*
 * ckks_ct_mul_relin_rescale_host with the host ciphertexts in the 48-bit wire
 * format (6 bytes per residue, 25 % less PCIe traffic both ways): a_host,
 * b_host hold 6 n_ct 2 level N bytes, out_host receives 6 n_ct 2 (level-1) N
 * bytes; unpacking and packing run on the GPU inside the call.  Workspace:
 * ckks_ct_mul_host48_workspace_bytes(ctx, chunk, level) bytes.  Replaces the
 * host side of scripts/verify_e2e_mult.py:78 e2e_mult for packed batches
 * (the reference moves vectors as $readmemh hex words, scripts/gen_ntt_vectors.py).
 */
size_t ckks_ct_mul_host48_workspace_bytes(const ckks_ctx* ctx, int chunk, int level);
int ckks_ct_mul_relin_rescale_host48(const ckks_ctx* ctx, void* out_host, const void* a_host,
                                     const void* b_host, const uint64_t* key, int n_ct, int level,
                                     int chunk, void* workspace, size_t workspace_bytes, void* stream);

/*
 * Stream-ordered forms of the two host-buffer calls above: the same chunked
 * H2D -> kernels -> D2H pipeline is enqueued (after the work already queued
 * on `stream`) and the call returns without waiting.  ckks_ct_mul_host_join
 * (stream) then makes `stream` wait for every chunk enqueued so far on the
 * current device; the outputs are in host memory once `stream` has reached
 * that point (cudaStreamSynchronize).  Host buffers and the workspace must
 * stay valid and unmodified until then; consecutive calls may share one
 * workspace (its slots are reused in stream order).  Back-to-back calls
 * overlap: the next call's input copies run while the previous call's last
 * chunks compute and copy back.  Like the blocking calls, they replace the
 * host side of scripts/verify_e2e_mult.py:78 e2e_mult for batches.
 */
int ckks_ct_mul_relin_rescale_host_async(const ckks_ctx* ctx, uint64_t* out_host, const uint64_t* a_host,
                                         const uint64_t* b_host, const uint64_t* key, int n_ct, int level,
                                         int chunk, void* workspace, size_t workspace_bytes, void* stream);
int ckks_ct_mul_relin_rescale_host48_async(const ckks_ctx* ctx, void* out_host, const void* a_host,
                                           const void* b_host, const uint64_t* key, int n_ct, int level,
                                           int chunk, void* workspace, size_t workspace_bytes, void* stream);
int ckks_ct_mul_host_join(void* stream);

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
 *  - Always one sub-batch on the caller's stream: CKKS_TUNE_CM_SPLIT and the
 *    default split of large batches are ignored here, since concurrent
 *    sub-batches run on internal streams and events created on first use.
 */
int ckks_ct_mul_relin_rescale_noalloc(const ckks_ctx* ctx, uint64_t* out, const uint64_t* ct_a,
                                      const uint64_t* ct_b, const uint64_t* key, int n_ct,
                                      int level, void* stream);

/*
 * Batched uneven workload in ONE persistent launch.  A bucket is n_ct
 * same-shape operations on one context (N = 2^12 or 2^13): op
 * CKKS_BATCH_CT_CT = ct_a x ct_b + relinearisation + rescale
 * (ckks_ct_mul_relin_rescale's operands: a, b ciphertexts [n_ct][2][level][N],
 * key prepared by ckks_relin_key_prepare, out [n_ct][2][level - 1][N]) or
 * CKKS_BATCH_CT_PT = ciphertext x plaintext + rescale
 * (ckks_ct_mul_plain_rescale's: b = plaintexts, one per ciphertext when
 * pt_per_ct, else one shared).  Results are bit-identical to those entry
 * points.
 *
 * ckks_batch_plan_create validates the buckets, allocates the plan's device
 * memory once (scratch for every ct x ct pair, the work list, dependency
 * counters) and lists every work unit (a pair's tensor limbs, ModUp target
 * primes, ModDown polynomials; a ct x pt item's two polynomials) in a
 * dependency-respecting order, each dependent stage lag_percent % of one
 * wave after its producers (0..10000; 400 is a good default), cut into
 * slots: one N = 2^13 unit for a whole 512-thread CTA, or two N = 2^12 units
 * that the CTA's halves run side by side.  The buckets' device pointers are
 * baked into the plan: they must stay valid while it is used.
 *
 * ckks_batch_plan_run zeroes the plan's counters (one memset) and launches
 * the persistent kernel on `stream`: CTAs take units from one atomic ticket;
 * a unit whose inputs are not finished waits on its item's counter with a
 * bounded spin of at most wait_cycles SM cycles (<= 0: 2^31 - 1).  On expiry
 * the kernel records it for ckks_device_status (CKKS_ETIMEOUT), stops every
 * CTA, and leaves the unfinished items incomplete.  Both calls of a run may
 * be captured into a CUDA graph (one memset node, one kernel node).  flags:
 * 0, CKKS_BATCH_RUN_PHASED (run the phased list instead of the paired one,
 * below), and / or CKKS_BATCH_RUN_UNMET_WAIT (a test hook: the ModUp units of
 * the first ct x ct item wait for one tensor unit more than exist, so that
 * wait ends only by its limit).
 *
 * The plan holds two lists of the same units.  The paired list (the
 * default): both ring sizes interleaved, N = 2^12 units two per slot, so the
 * two halves of a CTA finish together before it takes its next slot.  The
 * phased list: the N = 2^13 units first, one per whole-CTA slot, then every
 * N = 2^12 unit in a half slot of its own, which each half of each CTA takes
 * from a second ticket independently of the other half (its kernel is a
 * separate build; on B200 it measured 1-3 % slower at lags 200-800, the cost
 * of its larger register spills in the N = 2^13 units outweighing the
 * decoupled halves).  ckks_batch_plan_info reports the paired list's slot
 * count.
 *
 * ckks_batch_plan_incomplete synchronises the device and counts the items
 * of the last run whose output is not complete (bucket_complete, if not
 * NULL, gets one 0/1 byte per bucket).
 *
 * The reference batches by time-multiplexing four poly-mult instances on one
 * datapath (rtl/m4/e2e_ckks_mult_ctrl_m4.sv:368-482); it has no equivalent
 * of the uneven-shape work list.
 */
enum { CKKS_BATCH_CT_CT = 0, CKKS_BATCH_CT_PT = 1 };
enum { CKKS_BATCH_RUN_UNMET_WAIT = 1, CKKS_BATCH_RUN_PHASED = 2 };
typedef struct ckks_batch_bucket {
  const ckks_ctx* ctx;
  int32_t op;
  int32_t n_ct;
  int32_t level;
  int32_t pt_per_ct;
  const uint64_t* a;
  const uint64_t* b;
  uint64_t* out;
  const uint64_t* key;
} ckks_batch_bucket;
typedef struct ckks_batch_plan ckks_batch_plan;
int ckks_batch_plan_create(const ckks_batch_bucket* buckets, int n_buckets, int lag_percent,
                           ckks_batch_plan** plan);
int ckks_batch_plan_run(ckks_batch_plan* plan, long long wait_cycles, int flags, void* stream);
int ckks_batch_plan_incomplete(ckks_batch_plan* plan, int* n_incomplete, uint8_t* bucket_complete);
int ckks_batch_plan_info(const ckks_batch_plan* plan, long long* n_units, long long* n_slots, int* grid,
                         int* smem_bytes, size_t* device_bytes);
void ckks_batch_plan_destroy(ckks_batch_plan* plan);
/*
 * The plan's work list computed on the host alone (no device): for buckets
 * described by op, n_ct, level, log_n (12 or 13) and a cost that ranks them
 * (costliest first), with dependent stages `lag` units after their
 * producers, writes 4 x uint32 per slot: two units (bucket << 8 | stage << 6
 * | sub, item), stage 0 tensor (sub = limb), 1 ModUp (sub = target prime,
 * level = the special prime), 2 ModDown (sub = output polynomial), 3 ct x pt
 * (sub = output polynomial); the second unit is (0xFFFFFFFF, 0) in a slot of
 * one.  *n_slots: capacity in (at least the number of units), slots out.
 */
int ckks_batch_schedule(int n_buckets, const int* op, const int* n_ct, const int* level, const int* log_n,
                        const double* cost, long long lag, uint32_t* slots, long long* n_slots);
/* The phased list (CKKS_BATCH_RUN_PHASED) on the host alone: *n_whole
 * whole-CTA slots of one N = 2^13 unit each (dependent stages `lag` units
 * apart), then half slots of one N = 2^12 unit each (2 lag units apart); the
 * slot format above, every second unit (0xFFFFFFFF, 0). */
int ckks_batch_schedule_phased(int n_buckets, const int* op, const int* n_ct, const int* level, const int* log_n,
                               const double* cost, long long lag, uint32_t* slots, long long* n_slots,
                               long long* n_whole);

/*
 * Per-kernel device timing (tracing).  When enabled, the multi-kernel entry
 * points record CUDA events around each kernel on the launching stream;
 * ckks_profile_read(stage) resolves them and returns the accumulated device
 * milliseconds and launch count of a stage: 0 = ct-mult tensor, 1 = ct-mult
 * ModUp + key inner product, 2 = ct-mult ModDown + rescale, 3 = ckks_ntt,
 * 4 = other kernels, 5 = the fused ct-mult kernel, 6 = the persistent
 * batch kernel (ckks_batch_plan_run).
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
