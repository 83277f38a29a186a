"""RTL-flow file formats: $readmemh hex (with comments and @ directives),
decimal .mem vectors and modulus-chain JSON, read and written by
ckks_b200.formats; on the GPU, testbench vectors go through the NTT from
file to file and match the reference's golden outputs."""
import json
from pathlib import Path

import numpy as np
import pytest

GD = Path(__file__).resolve().parent / "golden"


def test_memh_round_trip_and_directives(tmp_path):
    from ckks_b200.formats import read_memh, write_memh
    vals = np.array([0, 1, 112, 0x1FFFFFFFFFFF, 35184371884032], dtype=np.uint64)
    write_memh(tmp_path / "v.hex", vals, width_bits=45)
    lines = (tmp_path / "v.hex").read_text().splitlines()
    assert all(len(l) == 12 for l in lines)
    assert np.array_equal(read_memh(tmp_path / "v.hex"), vals)
    (tmp_path / "d.hex").write_text("// ROM\n@2\n0a 0b // two words\n@0\n01\n")
    assert read_memh(tmp_path / "d.hex").tolist() == [1, 0, 10, 11]
    with pytest.raises(ValueError):
        write_memh(tmp_path / "x.hex", [8], width_bits=3)


def test_chain_json(tmp_path):
    from ckks_b200.formats import load_chain
    chain = json.load(open(GD / "golden_core.json"))["chain4"]
    p = tmp_path / "chain.json"
    p.write_text(json.dumps([{"q": r["q"], "omega": r["omega"], "N": r["N"]} for r in chain]))
    back = load_chain(p)
    assert [r["q"] for r in back] == [r["q"] for r in chain]


@pytest.mark.gpu
def test_transform_files_match_golden(cuda, tmp_path):
    from ckks_b200.context import Context
    from ckks_b200.formats import context_from_chain, read_memh, transform_file, write_memh
    from oracle.ntt import ntt_dit
    arr = np.load(GD / "golden_core.npz")
    toy = json.load(open(GD / "golden_core.json"))["toy"]
    ctx = Context.get(4, [toy["q"]], omega=[toy["omega"]])
    src = tmp_path / "ntt_in_all.mem"
    src.write_text("".join(f"{int(v)}\n" for v in arr["toy_ntt_in"].reshape(-1)))
    out = transform_file(ctx, src, tmp_path / "ntt_out_all.mem")
    assert np.array_equal(out.reshape(arr["toy_ntt_out"].shape), arr["toy_ntt_out"])
    write_memh(tmp_path / "fwd.hex", out, width_bits=7)
    back = transform_file(ctx, tmp_path / "fwd.hex", tmp_path / "back.hex", inverse=True)
    assert np.array_equal(back.reshape(arr["toy_ntt_in"].shape), arr["toy_ntt_in"])
    assert np.array_equal(read_memh(tmp_path / "back.hex"), back)
    # a chain context (N = 16384 roots taken down to N = 4096)
    chain = json.load(open(GD / "golden_core.json"))["chain4"]
    cctx = context_from_chain(chain, 12)
    rng = np.random.default_rng(0)
    q1, om = int(chain[1]["q"]), pow(int(chain[1]["omega"]), 4, int(chain[1]["q"]))
    a = rng.integers(0, q1, 4096).astype(np.uint64)
    write_memh(tmp_path / "a.hex", a)
    got = transform_file(cctx, tmp_path / "a.hex", tmp_path / "A.hex", prime=1)
    assert got.tolist() == ntt_dit([int(v) for v in a], om, q1)


def test_pack48_host_round_trip():
    import torch
    from ckks_b200 import ops
    x = torch.tensor([0, 1, (1 << 47) - 1, 35184371884033, 0x123456789ABC], dtype=torch.int64).view(torch.uint64)
    b = ops.pack48_host(x)
    assert b.numel() == 30 and b[:6].tolist() == [0] * 6 and b[6:12].tolist() == [1, 0, 0, 0, 0, 0]
    assert torch.equal(ops.unpack48_host(b, x.shape), x)
