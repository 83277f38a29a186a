"""Generate golden vectors by running the reference's own Python functions.

Run where a checkout of the reference project exists (read-only is fine),
naming its root in REFERENCE_ROOT (required; there is no default):

    REFERENCE_ROOT=<reference checkout> python tests/golden/make_golden.py

It imports the reference's golden-model functions by path (never copying
their source), runs them on seeded inputs and writes the inputs/outputs to
tests/golden/*.npz / *.json.  The committed outputs are what the tests compare
the oracle and the GPU path against; the reference itself is not needed at
test time.  tb/ref/gen_ntt_reference.py executes file-writing code at import,
so it is executed in a temporary copy of its directory and its .mem outputs
are read back.
"""
from __future__ import annotations

import hashlib
import importlib.util
import json
import os
import random
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent


def _reference_root() -> Path:
    root = os.environ.get("REFERENCE_ROOT")
    if not root:
        raise SystemExit("make_golden.py: set REFERENCE_ROOT to the reference project's checkout")
    path = Path(root)
    if not (path / "scripts").is_dir():
        raise SystemExit(f"make_golden.py: {path} has no scripts/ directory; is it the reference checkout?")
    return path


REF = _reference_root() if __name__ == "__main__" else Path(os.environ.get("REFERENCE_ROOT", "."))


def load(relpath: str, name: str):
    spec = importlib.util.spec_from_file_location(name, REF / relpath)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod  # dataclasses look their module up here
    import contextlib
    import io
    try:
        with contextlib.redirect_stdout(io.StringIO()):
            spec.loader.exec_module(mod)
    except SystemExit:
        pass  # some scripts run their checks at import and exit; their functions are defined first
    return mod


def sha(vals) -> str:
    h = hashlib.sha256()
    for v in vals:
        h.update(int(v).to_bytes(16, "little", signed=True))
    return h.hexdigest()


def read_hex(relpath: str) -> list[int]:
    with open(REF / relpath) as f:
        return [int(l, 16) for l in f if l.strip()]


def main() -> int:
    arrays: dict[str, np.ndarray] = {}
    meta: dict = {"reference": "YI-HAIBO/cipher-pu", "generator": "tests/golden/make_golden.py"}

    # ---------------------------------------------------------------- 1 gen_ntt_reference (N=16, q=113)
    with tempfile.TemporaryDirectory() as td:
        tdir = Path(td) / "tbref"
        tdir.mkdir()
        shutil.copy(REF / "tb/ref/gen_ntt_reference.py", tdir / "gen_ntt_reference.py")
        subprocess.run([sys.executable, "gen_ntt_reference.py"], cwd=tdir, check=True,
                       capture_output=True)
        ins, outs = [], []
        for v in range(10):
            ins.append([int(l) for l in open(tdir / "ref" / f"ntt_input_{v}.mem") if l.strip()])
            outs.append([int(l) for l in open(tdir / "ref" / f"ntt_output_{v}.mem") if l.strip()])
    arrays["toy_ntt_in"] = np.array(ins, dtype=np.uint64)
    arrays["toy_ntt_out"] = np.array(outs, dtype=np.uint64)
    meta["toy"] = {"N": 16, "q": 113, "omega": 40, "omega_inv": 65, "n_inv": 106,
                   "source": "tb/ref/gen_ntt_reference.py:78 ntt (seeds 42+v)"}

    # ---------------------------------------------------------------- 2 gen_omega_tables on q3 / N=4096
    got = load("scripts/gen_omega_tables.py", "ref_got")
    q3 = 17592186175489
    tw = read_hex("rtl/m5/tw/tw_omega_q3_n4096.hex")
    twi = read_hex("rtl/m5/tw/tw_omegainv_q3_n4096.hex")
    omega = tw[1]
    omega_inv = twi[1]
    n = 4096
    tab = got.generate_table(omega, q3, n)
    assert tab == tw, "generate_table disagrees with committed hex"
    rng = random.Random(0xC77)
    a = [rng.randint(0, q3 - 1) for _ in range(n)]
    ah = got._ntt_dit(a, omega, q3)
    rec = got._intt_dif(ah, omega_inv, pow(n, -1, q3), q3)
    assert rec == a
    arrays["q3_ntt_in"] = np.array(a, dtype=np.uint64)
    arrays["q3_ntt_out"] = np.array(ah, dtype=np.uint64)
    meta["q3"] = {"q": q3, "N": n, "omega": omega, "omega_inv": omega_inv,
                  "n_inv": pow(n, -1, q3), "tw_sha": sha(tw), "twinv_sha": sha(twi),
                  "tw_len": len(tw), "source": "scripts/gen_omega_tables.py:96,154,188; rtl/m5/tw/tw_omega*_q3_n4096.hex"}
    errs = got.verify(n, q3, omega, omega_inv, tab, got.generate_table(omega_inv, q3, n))
    meta["q3"]["verify_errors"] = errs

    # committed chain4 fixtures: constants + table digests
    chain = json.load(open(REF / "rtl/m2/modulus_chain_chain4.json"))
    meta["chain4"] = []
    for i, rec in enumerate(chain):
        t = read_hex(f"rtl/m2/omega_table_chain4_q{i}.hex")
        ti = read_hex(f"rtl/m2/omega_inv_table_chain4_q{i}.hex")
        meta["chain4"].append({k: rec[k] for k in ("q", "primitive_root", "omega", "omega_inv", "N", "N_INV")}
                              | {"tw_sha": sha(t), "twinv_sha": sha(ti), "tw_len": len(t),
                                 "tw_head": t[:4], "twinv_head": ti[:4]})
    # RNS p1/p2/p3 tables (N=16, 4096): digests + head
    meta["rns_tw"] = {}
    for tag in ("p1", "p2", "p3", "q3", "toy"):
        for nn in (8, 16, 4096, 16384):
            for kind in ("omega", "omegainv"):
                rel = f"rtl/m5/tw/tw_{kind}_{tag}_n{nn}.hex"
                if (REF / rel).exists():
                    t = read_hex(rel)
                    meta["rns_tw"][f"{kind}_{tag}_n{nn}"] = {"sha": sha(t), "len": len(t), "head": t[:4]}

    # ---------------------------------------------------------------- 3 gen_poly_mult_vectors_n12 (cyclic)
    pm = load("tb/ref/gen_poly_mult_vectors_n12.py", "ref_pm12")
    vecs = pm.build_vectors()
    pm_meta = []
    for i, (tag, a, b) in enumerate(vecs):
        c = pm.poly_mult_via_ntt(a, b, pm.N, pm.Q, pm.OMEGA, pm.OMEGA_INV)
        pm_meta.append({"tag": tag, "c_sha": sha(c), "c_head": c[:4]})
        if tag in ("rand0", "sparse"):
            arrays[f"pm12_{tag}_a"] = np.array(a, dtype=np.uint64)
            arrays[f"pm12_{tag}_b"] = np.array(b, dtype=np.uint64)
            arrays[f"pm12_{tag}_c"] = np.array(c, dtype=np.uint64)
    meta["pm12"] = {"q": pm.Q, "N": pm.N, "psi": pm.PSI, "omega": pm.OMEGA, "omega_inv": pm.OMEGA_INV,
                    "n_inv": pm.N_INV, "vectors": pm_meta,
                    "source": "tb/ref/gen_poly_mult_vectors_n12.py:103,149"}

    # ---------------------------------------------------------------- 4 verify_keyswitch (negacyclic)
    vk = load("scripts/verify_keyswitch.py", "ref_vk")
    q0 = vk.load_chain()[0]["q"]
    rng = random.Random(42)
    cases = []
    for n_toy in (16, 64):
        for t in range(3):
            e0, e1, e2, ka = ([rng.randrange(q0) for _ in range(n_toy)] for _ in range(4))
            s = [rng.randrange(q0) for _ in range(n_toy)]
            e_ks = [rng.randrange(100) for _ in range(n_toy)]
            kb = vk.poly_add(vk.poly_mult(ka, s, q0), e_ks, q0)
            f0, f1 = vk.relin(e0, e1, e2, ka, kb, q0)
            cases.append([e0, e1, e2, ka, kb, f0, f1])
    arrays["relin16"] = np.array([c for c in cases[:3]], dtype=np.uint64)
    arrays["relin64"] = np.array([c for c in cases[3:]], dtype=np.uint64)
    # negacyclic poly_mult at N=256 on the 45-bit config prime and on the toy q=113
    qc = 35184371884033
    rng = random.Random(7)
    a = [rng.randrange(qc) for _ in range(256)]
    b = [rng.randrange(qc) for _ in range(256)]
    arrays["pmneg256"] = np.array([a, b, vk.poly_mult(a, b, qc)], dtype=np.uint64)
    a = [rng.randrange(113) for _ in range(16)]
    b = [rng.randrange(113) for _ in range(16)]
    arrays["pmneg16_q113"] = np.array([a, b, vk.poly_mult(a, b, 113)], dtype=np.uint64)
    meta["keyswitch"] = {"q": q0, "config_prime": qc,
                         "source": "scripts/verify_keyswitch.py:48 poly_mult, :62 relin"}

    # ---------------------------------------------------------------- 5 verify_rescale
    vr = load("scripts/verify_rescale.py", "ref_vr")
    primes = [p["q"] for p in vr.load_chain()]
    rs = {}
    for i in range(len(primes) - 1):
        qi, qo = primes[i], primes[i + 1]
        pts = [0, 1, 2, qi - 3, qi - 2, qi - 1, qo - 1, qo, qo + 1]
        pts = sorted({p for p in pts if 0 <= p < qi})
        rng = random.Random(1000 + i)
        pts += [rng.randrange(qi) for _ in range(2000)]
        arrays[f"rescale_{i}_in"] = np.array(pts, dtype=np.uint64)
        arrays[f"rescale_{i}_out"] = np.array([vr.rescale_coeff(c, qi, qo) for c in pts], dtype=np.uint64)
    rng = random.Random(12345)
    poly = [rng.randrange(primes[0]) for _ in range(vr.N)]
    outp = vr.rescale_poly(poly, primes[0], primes[1])
    arrays["rescale_poly_out"] = np.array(outp, dtype=np.uint64)
    meta["rescale"] = {"primes": primes, "poly_seed": 12345, "N": vr.N,
                       "source": "scripts/verify_rescale.py:38,56,101"}

    # ---------------------------------------------------------------- 6 verify_e2e_mult
    ve = load("scripts/verify_e2e_mult.py", "ref_ve")
    ch = ve.load_chain()
    qi, qo = ch[0]["q"], ch[1]["q"]
    rng = random.Random(42)
    e2e = []
    for t in range(4):
        c = [[rng.randrange(qi) for _ in range(16)] for _ in range(6)]
        f0, f1 = ve.e2e_mult(c[0], c[1], c[2], c[3], c[4], c[5], qi, qo, ve.SCALE_BITS)
        e2e.append(c + [f0, f1])
    arrays["e2e16"] = np.array(e2e, dtype=np.uint64)
    rng = random.Random(5)
    xs = [rng.randrange(qi) for _ in range(4000)] + [0, 1, qi - 1]
    arrays["e2e_rescale_in"] = np.array(xs, dtype=np.uint64)
    arrays["e2e_rescale_out"] = np.array([ve.rescale(x, qi, qo, ve.SCALE_BITS) for x in xs], dtype=np.uint64)
    meta["e2e"] = {"q_in": qi, "q_out": qo, "scale_bits": ve.SCALE_BITS,
                   "source": "scripts/verify_e2e_mult.py:70 rescale, :78 e2e_mult"}

    # ---------------------------------------------------------------- 7 _verify_fastred (b * omega mod q3)
    fr = load("scripts/_verify_fastred.py", "ref_fr")
    rng = random.Random(20261003)
    bw = [(rng.randrange(fr.Q), rng.randrange(fr.Q)) for _ in range(4096)]
    arrays["fastred_b"] = np.array([b for b, _ in bw], dtype=np.uint64)
    arrays["fastred_w"] = np.array([w for _, w in bw], dtype=np.uint64)
    arrays["fastred_out"] = np.array([fr.fast_red(b * w) for b, w in bw], dtype=np.uint64)
    meta["fastred"] = {"q": fr.Q, "source": "scripts/_verify_fastred.py:55 fast_red (seed 20261003)"}

    # ---------------------------------------------------------------- 8 golden_fc_layer
    sys.path.insert(0, str(REF / "scripts"))
    fc = load("scripts/golden_fc_layer.py", "ref_fc")
    import contextlib
    import io
    with contextlib.redirect_stdout(io.StringIO()):
        f1, f2 = fc.build_mnist_cnn_model(512, 128, 10)
        y1, y1q = f1.test_forward(num_slots=4)
        y2, y2q = f2.test_forward(num_slots=4)
    arrays["fc1_w"] = f1.weights
    arrays["fc2_w"] = f2.weights
    arrays["fc1_test_y"] = np.asarray(y1, dtype=np.float64)
    arrays["fc2_test_y"] = np.asarray(y2, dtype=np.float64)
    arrays["fc1_test_yq"] = np.asarray(y1q, dtype=np.float64)
    rng = np.random.default_rng(99)
    xe = rng.standard_normal((4, 512))
    arrays["fc_e2e_x"] = xe
    arrays["fc_e2e_logits"] = np.asarray(f2.forward(np.maximum(f1.forward(xe), 0)), dtype=np.float64)
    meta["fc"] = {"source": "scripts/golden_fc_layer.py:28,93,128"}

    # ---------------------------------------------------------------- 9 slot encode / decode
    ms = load("scripts/verify_multi_slot_simd.py", "ref_ms")
    rng = np.random.default_rng(3)
    vv = rng.uniform(-1, 1, size=(5, ms.SLOTS))
    arrays["simd_v"] = vv
    arrays["simd_m"] = np.array([ms.encode(v) for v in vv])
    arrays["simd_dec"] = np.array([ms.decode(ms.encode(v)) for v in vv])
    mlp = load("scripts/verify_project_b_mlp_reference.py", "ref_mlp")
    xs = rng.standard_normal((3, 64)) + 1j * rng.standard_normal((3, 64))
    arrays["negfft_x"] = xs
    arrays["negfft_y"] = np.array([mlp.neg_fft(x) for x in xs])
    arrays["negifft_y"] = np.array([mlp.neg_ifft(x) for x in xs])
    meta["simd"] = {"N": ms.N_POLY, "scale": ms.SCALE, "slots": ms.SLOTS,
                    "source": "scripts/verify_multi_slot_simd.py:32,42,75,88; "
                              "scripts/verify_project_b_mlp_reference.py:60,73"}

    # ---------------------------------------------------------------- 10 noise monitor
    mh = load("scripts/verify_m4_h_multilayer.py", "ref_mh")
    rng = random.Random(11)
    nm = []
    for q, n, mag in ((q3, 4096, None), (q0, 1024, 1 << 20), (113, 16, None)):
        c = [rng.randrange(q) if mag is None else (rng.randrange(-mag, mag) % q) for _ in range(n)]
        e, r = mh.noise_monitor_energy(c, q)
        sw, rw = mh.layer_sigma_welford(c, q)
        nm.append({"q": q, "coeffs": c, "E": e, "r_hat": r, "sigma_w": sw, "r_hat_w": rw})
    meta["noise"] = {"cases": nm, "source": "scripts/verify_m4_h_multilayer.py:162,193"}

    # ---------------------------------------------------------------- 11 gear controllers
    ad = load("scripts/verify_m4_h_adaptive.py", "ref_ad")
    ga = load("scripts/verify_m4_a_gear_ctrl.py", "ref_ga")
    rs = [10 ** (-k / 4) for k in range(0, 40)]
    seq_r = [0.001, 0.001, 0.3, 0.001, 0.2, 0.05, 0.05, 0.05, 0.4, 0.01, 0.01, 0.01, 0.01]
    hyst = []
    g_old = 0
    for r in seq_r:
        g_new = ad.select_gear_safe(r)
        g_old = ad.select_gear_with_hysteresis(g_new, g_old, r)
        hyst.append(g_old)
    agc = mlp.AdaptiveGearCtrl()
    agc_seq = [agc.step(r) for r in [0.05, 0.05, 0.05, 0.3, 0.3, 0.3, 0.15, 0.15, 0.15, 0.6, 0.6, 0.6]]
    meta["gear"] = {
        "geo": [{k: g[k] for k in ("threshold", "trunc_bits", "skip_rate")} | {
            "extra": ad.compute_extra(g)[2], "total_growth": ad.total_growth(g)} for g in ad.GEO],
        "r_sweep": rs, "safe": [ad.select_gear_safe(r) for r in rs],
        "seq_r": seq_r, "hyst": hyst,
        "gear_config": [ga.get_gear_config(g) for g in range(6)],
        "gear_config_ovr": ga.get_gear_config(2, 1234, True),
        "agc_seq": agc_seq,
        "source": "scripts/verify_m4_h_adaptive.py:37,48,101,114; scripts/verify_m4_a_gear_ctrl.py:41; "
                  "scripts/verify_project_b_mlp_reference.py:279"}

    # ---------------------------------------------------------------- 12 block sparsity
    da = load("scripts/verify_m4_d_approx_mult.py", "ref_da")
    rng = random.Random(5)
    bs = []
    for B in (1, 2, 4, 16):
        x = [rng.randrange(113) for _ in range(16)]
        out, skipped = da.post_process_block(x, 20, True, 113, B)
        bs.append({"B": B, "x": x, "out": out, "skipped": skipped})
    meta["block_post"] = bs
    e10 = load("scripts/exp_e10_sparsity_sweep_v2.py", "ref_e10")
    rng = np.random.default_rng(4)
    W = rng.standard_normal((128, 784)) / np.sqrt(784)
    for thr in (0.02, 0.05):
        mW, skip, tot, dens = e10.apply_block_sparse_mask(W, thr, 4)
        arrays[f"bsm_mask_{thr}"] = np.packbits(mW != 0)
        meta[f"bsm_{thr}"] = {"skip": skip, "total": tot, "density": dens}
    arrays["bsm_W"] = W
    meta["block_sparse_source"] = ("scripts/verify_m4_d_approx_mult.py:50 post_process_block; "
                                   "scripts/exp_e10_sparsity_sweep_v2.py:102 apply_block_sparse_mask")

    # ---------------------------------------------------------------- 13 DARE (exp_e24)
    e24 = load("scripts/exp_e24_rotation_bootstrap.py", "ref_e24")
    n24, q24 = e24.N, e24.Q
    rng = np.random.default_rng(8)
    s = rng.integers(-1, 2, size=n24)
    np.random.seed(1234)
    m_int = rng.integers(-(1 << 20), 1 << 20, size=n24)
    e0 = rng.integers(-3, 4, size=n24)
    ct = e24.rlwe_encrypt_mint(m_int, s, e0, q24)
    dec = e24.decrypt_exact_int(ct, s, q24)
    ct2, m_new = e24.reencrypt(ct, s, q24, 2 ** 20, np.random.default_rng(9))
    dec2 = e24.decrypt_exact_int(ct2, s, q24)
    arrays["dare_s"] = s
    arrays["dare_ct_b"] = np.asarray(ct[0], dtype=np.int64)
    arrays["dare_ct_a"] = np.asarray(ct[1], dtype=np.int64)
    arrays["dare_dec"] = dec
    arrays["dare_ct2_b"] = np.asarray(ct2[0], dtype=np.int64)
    arrays["dare_ct2_a"] = np.asarray(ct2[1], dtype=np.int64)
    arrays["dare_dec2"] = dec2
    arrays["dare_m_new"] = np.asarray(m_new, dtype=np.int64)
    arrays["dare_e_new"] = np.random.default_rng(9).integers(-1, 2, size=n24).astype(np.int64)
    meta["dare"] = {"N": n24, "q": q24, "source": "scripts/exp_e24_rotation_bootstrap.py:126,209,287"}

    np.savez_compressed(OUT / "golden_core.npz", **arrays)
    with open(OUT / "golden_core.json", "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("wrote", OUT / "golden_core.npz", sum(a.nbytes for a in arrays.values()), "bytes raw")
    return 0


def rotation_vectors() -> int:
    """Automorphism and monomial-product goldens from
    scripts/exp_e24_rotation_bootstrap.py:143 automorphism_exact, :167
    automorphism_key_exact and :189 poly_mul_x_power -> golden_rot.npz/json."""
    cwd = os.getcwd()
    try:
        e24 = load("scripts/exp_e24_rotation_bootstrap.py", "ref_e24")
    finally:
        os.chdir(cwd)  # the module changes directory at import
    arrays: dict[str, np.ndarray] = {}
    cases = []
    rng = np.random.default_rng(2024)
    for n, q, nus in ((16, 113, (3, 5, 4, 0, 31, 17)),
                      (1024, 998244353, (5, 2047, 6, 1025, 3 * 1024 + 7)),
                      (4096, 35184371884033, (5, 25, 8191, 12, 4097))):
        c0 = rng.integers(0, q, n).astype(np.int64)
        c1 = rng.integers(0, q, n).astype(np.int64)
        for nu in nus:
            g0, g1 = e24.automorphism_exact((c0, c1), nu, n, q)
            tag = f"aut_{n}_{nu}"
            arrays[tag + "_in"] = np.stack([c0, c1]).astype(np.uint64)
            arrays[tag + "_out"] = np.stack([np.asarray(g0), np.asarray(g1)]).astype(np.int64).astype(np.uint64)
            cases.append({"kind": "automorphism_exact", "n": n, "q": q, "nu": nu, "key": tag})
        for nu in (0, 1, 7, n // 2, n - 1):
            out = e24.poly_mul_x_power(c0, nu, n, q)
            tag = f"mono_{n}_{nu}"
            arrays[tag + "_in"] = c0.astype(np.uint64)
            arrays[tag + "_out"] = np.asarray(out).astype(np.int64).astype(np.uint64)
            cases.append({"kind": "poly_mul_x_power", "n": n, "q": q, "nu": nu, "key": tag})
    s = rng.integers(-1, 2, 1024)
    ks = e24.automorphism_key_exact(s, 5, 1024, 998244353)
    arrays["autkey_in"] = s.astype(np.int64)
    arrays["autkey_out"] = np.asarray(ks).astype(np.int64).astype(np.uint64)
    cases.append({"kind": "automorphism_key_exact", "n": 1024, "q": 998244353, "nu": 5, "key": "autkey"})
    np.savez_compressed(OUT / "golden_rot.npz", **arrays)
    with open(OUT / "golden_rot.json", "w") as f:
        json.dump({"reference": "YI-HAIBO/cipher-pu", "generator": "tests/golden/make_golden.py --only rot",
                   "source": "scripts/exp_e24_rotation_bootstrap.py:143,167,189", "cases": cases}, f, indent=1)
    print("wrote", OUT / "golden_rot.npz")
    return 0


def activation_vectors() -> int:
    """Degree-5 Chebyshev activation fits of scripts/golden_activation.py
    (ActivationGoldenModel: _fit_piecewise_chebyshev, approximate) with one
    segment on [-1, 1] (the form a homomorphic polynomial can evaluate) and the
    reference's default two segments -> golden_act.json."""
    act = load("scripts/golden_activation.py", "ref_golden_activation")
    out = {"reference": "YI-HAIBO/cipher-pu", "generator": "tests/golden/make_golden.py --only act",
           "source": "scripts/golden_activation.py:28 ActivationGoldenModel", "models": {}}
    xs = np.linspace(-1, 0.999, 41)
    for segs in (1, 2):
        g = act.ActivationGoldenModel(poly_order=5, num_segments=segs)
        m = {}
        for name in ("sigmoid", "tanh", "relu"):
            m[name] = {"segments": g.coeffs[name], "x": xs.tolist(),
                       "approx": [float(v) for v in g.approximate(xs.copy(), name)],
                       "exact": [float(v) for v in g.evaluate(xs.copy(), name)]}
        out["models"][f"order5_segments{segs}"] = m
    with open(OUT / "golden_act.json", "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", OUT / "golden_act.json")
    return 0


def convgap_vectors() -> int:
    """Inner-product / Conv + GAP goldens from
    scripts/exp_e24_rotation_bootstrap.py:241 scatter_w, :136 mul_plain_exact,
    :109 decrypt_exact, :263 inner_product, :278 coef_sum, :307 enc_msg and
    :615 encrypted_inference_fused (ConvGAPNet without ReLU, seeded random
    initialisation, synthetic images) -> golden_convgap.npz/json."""
    import torch
    cwd = os.getcwd()
    try:
        e24 = load("scripts/exp_e24_rotation_bootstrap.py", "ref_e24")
    finally:
        os.chdir(cwd)
    n, q, scale = e24.N, e24.Q, e24.SCALE
    arrays: dict[str, np.ndarray] = {}
    meta = {"reference": "YI-HAIBO/cipher-pu", "generator": "tests/golden/make_golden.py --only convgap",
            "source": "scripts/exp_e24_rotation_bootstrap.py:109,136,241,263,278,307,615",
            "N": n, "q": q, "scale": scale, "scatter": [], "inner": [], "fused": []}
    rng = np.random.default_rng(4040)
    # scatter_w: index 0 (negated), repeats, indices past N (wrap), half-way roundings
    sc_cases = [(list(range(10)), rng.uniform(-1, 1, 10)),
                ([0, 0, 5, 5, 5, 1023, 1024, 2049], [0.25, -0.5, 1.0, 2.0 / scale, 1.5 / scale,
                                                     -2.5 / scale, 0.75, -1.0]),
                (list(rng.integers(0, 784, 300)), rng.normal(0, 0.3, 300))]
    for k, (idx, w) in enumerate(sc_cases):
        m_w = e24.scatter_w([int(i) for i in idx], np.asarray(w, dtype=np.float64), scale, q, n)
        arrays[f"sc{k}_idx"] = np.asarray(idx, dtype=np.int64)
        arrays[f"sc{k}_w"] = np.asarray(w, dtype=np.float64)
        arrays[f"sc{k}_out"] = np.asarray(m_w, dtype=np.int64).astype(np.uint64)
        meta["scatter"].append(f"sc{k}")
    # mul_plain_exact and decrypt_exact on a uniform ciphertext
    s = rng.integers(-1, 2, n).astype(np.int64)
    arrays["s"] = s
    b = rng.integers(0, q, n).astype(np.int64)
    a = rng.integers(0, q, n).astype(np.int64)
    pb, pa = e24.mul_plain_exact((b, a), arrays["sc2_out"].astype(np.int64), q)
    arrays["mp_in"] = np.stack([b, a]).astype(np.uint64)
    arrays["mp_out"] = np.stack([np.asarray(pb), np.asarray(pa)]).astype(np.int64).astype(np.uint64)
    arrays["mp_dec"] = np.asarray(e24.decrypt_exact_int((pb, pa), s, q), dtype=np.int64)
    # inner_product / coef_sum on encrypted messages
    for k, dim in enumerate((16, 100, 784)):
        np.random.seed(500 + k)
        x = rng.uniform(0, 1, dim)
        w = rng.normal(0, 0.5, dim)
        e = rng.integers(-1, 2, n).astype(np.int64)
        ctb, cta = e24.enc_msg(x, s, e, q, scale)
        arrays[f"ip{k}_ct"] = np.stack([np.asarray(ctb), np.asarray(cta)]).astype(np.int64).astype(np.uint64)
        arrays[f"ip{k}_w"] = w
        meta["inner"].append({"key": f"ip{k}", "dim": dim,
                              "inner_product": e24.inner_product((ctb, cta), w, s, q, scale),
                              "coef_sum": e24.coef_sum((ctb, cta), dim, s, q, scale),
                              "plain_dot": float(np.dot(x, w)), "plain_sum": float(np.sum(x))})
    # fused Conv + GAP inference (noise argument 1 as the reference's run uses)
    torch.manual_seed(0)
    model = e24.ConvGAPNet(use_relu=False)
    arrays["conv_w"] = model.conv1.weight.detach().numpy().astype(np.float64)
    arrays["conv_b"] = model.conv1.bias.detach().numpy().astype(np.float64)
    arrays["fc_w"] = model.fc1.weight.detach().numpy().astype(np.float64)
    arrays["fc_b"] = model.fc1.bias.detach().numpy().astype(np.float64)
    for k in range(3):
        x = rng.uniform(0, 1, 784)
        np.random.seed(900 + k)
        logits, mc = e24.encrypted_inference_fused(model, x, s, q, scale, 1, np.random.default_rng(700 + k))
        np.random.seed(900 + k)
        e = np.random.default_rng(700 + k).integers(-1, 2, size=n).astype(np.int64)
        ctb, cta = e24.enc_msg(x, s, e, q, scale)
        with torch.no_grad():
            plain = model(torch.tensor(x, dtype=torch.float32).reshape(1, 1, 28, 28)).numpy()[0]
        arrays[f"fu{k}_x"] = x
        arrays[f"fu{k}_ct"] = np.stack([np.asarray(ctb), np.asarray(cta)]).astype(np.int64).astype(np.uint64)
        arrays[f"fu{k}_logits"] = np.asarray(logits, dtype=np.float64)
        arrays[f"fu{k}_plain"] = plain.astype(np.float64)
        meta["fused"].append({"key": f"fu{k}", "mult_count": int(mc)})
    np.savez_compressed(OUT / "golden_convgap.npz", **arrays)
    with open(OUT / "golden_convgap.json", "w") as f:
        json.dump(meta, f, indent=1)
    print("wrote", OUT / "golden_convgap.npz")
    return 0


if __name__ == "__main__":
    if sys.argv[1:] == ["--only", "convgap"]:
        sys.exit(convgap_vectors())
    if sys.argv[1:] == ["--only", "rot"]:
        sys.exit(rotation_vectors())
    if sys.argv[1:] == ["--only", "act"]:
        sys.exit(activation_vectors())
    rc = main()
    sys.exit(rc or rotation_vectors() or activation_vectors() or convgap_vectors())
