"""Key-material checkpoint (Evaluator.save_keys / load_keys): a fresh
evaluator that loads the file holds the same secret, relinearisation key and
Galois keys (raw and prepared, bit for bit), decrypts the first evaluator's
ciphertexts, gives bit-identical ct-mult and rotation results, and draws the
same randomness next (the sampler's stream counter travels with the keys).
A file of another schema or parameter set is refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pair(cuda, tmp_path_factory):
    import torch
    from ckks_b200.evaluator import Evaluator
    from ckks_b200.params import CkksParams
    P = CkksParams.standard(12, 3, seed=11)
    ev = Evaluator(P)
    ev.keygen()
    ev.galois_key(5)
    rng = np.random.default_rng(3)
    x = ev.encrypt_values(torch.from_numpy(rng.uniform(-1, 1, (2, 2048))))
    y = ev.encrypt_values(torch.from_numpy(rng.uniform(-1, 1, (2, 2048))))
    path = tmp_path_factory.mktemp("keys") / "keys.npz"
    ev.save_keys(path)
    ev2 = Evaluator(P)
    ev2.load_keys(path)
    return ev, ev2, x, y, path


def test_loaded_keys_are_identical(pair):
    import torch
    ev, ev2, _, _, _ = pair
    assert torch.equal(ev.sk.s_coef, ev2.sk.s_coef)
    assert torch.equal(ev.sk.s_eval, ev2.sk.s_eval)
    assert torch.equal(ev.ksk, ev2.ksk) and torch.equal(ev.rlk, ev2.rlk)
    assert sorted(ev.galois) == sorted(ev2.galois) == [5]
    assert torch.equal(ev.galois[5][0], ev2.galois[5][0]) and torch.equal(ev.galois[5][1], ev2.galois[5][1])


def test_loaded_keys_evaluate_bit_identically(pair):
    import torch
    ev, ev2, x, y, _ = pair
    assert torch.equal(ev.decrypt_coef(x), ev2.decrypt_coef(x))
    assert torch.equal(ev.mul_relin_rescale(x, y).data, ev2.mul_relin_rescale(x, y).data)
    assert torch.equal(ev.rotate(x, 5).data, ev2.rotate(x, 5).data)


def test_sampler_resumes_where_it_stopped(pair):
    import torch
    ev, ev2, _, _, path = pair
    from ckks_b200.evaluator import Evaluator
    ev3 = Evaluator(ev.params)
    ev3.load_keys(path)
    # ev2 and ev3 both resumed from the saved counter: the same next draws
    assert torch.equal(ev2.uniform(2, 3), ev3.uniform(2, 3))
    assert torch.equal(ev2.dgauss((1, ev.n)), ev3.dgauss((1, ev.n)))


def test_refuses_other_parameters_and_schemas(pair, tmp_path):
    from ckks_b200.evaluator import Evaluator
    from ckks_b200.params import CkksParams
    ev, _, _, _, path = pair
    other = Evaluator(CkksParams.standard(12, 3, seed=12))
    with pytest.raises(ValueError, match="another parameter set"):
        other.load_keys(path)
    z = dict(np.load(path))
    z["schema"] = np.int64(99)
    bad = tmp_path / "bad.npz"
    np.savez(bad, **z)
    with pytest.raises(ValueError, match="schema"):
        Evaluator(ev.params).load_keys(bad)
    with pytest.raises(ValueError, match="keygen"):
        Evaluator(ev.params).save_keys(tmp_path / "none.npz")
