"""BFV decryption through fast base conversion on the device (pg_bfv_decrypt):
equal to the oracle's DcrtGlweSecretKey::decrypt_inplace
(primus_fhe_core/src/secret_key/glwe.rs:782-837) on the same ciphertexts, and
to the encrypted messages."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("log_n,L,k,t,gamma,batch", [(10, 2, 1, 12289, 2199023190017, 3), (11, 1, 1, 16, 257, 2),
                                                      (9, 3, 2, 65537, 2199023190017, 2), (12, 10, 1, 3, 1 << 30 | 1, 1)])
def test_decrypt_matches_oracle(gpu, log_n, L, k, t, gamma, batch):
    n = 1 << log_n
    moduli = O.ntt_primes(1 << 54 if L == 1 else 1 << 50, 2 * n, L)
    tab = O.DcrtTable(log_n, moduli)
    base = O.RnsBase(moduli)
    lat = O.Lattice(tab, base, O.GadgetBasis(base, 20))
    sk = np.concatenate([lat.ternary(3, 10 + i) for i in range(k)])
    sk_ntt = tab.forward(sk.copy())
    msgs, cts = [], []
    for b in range(batch):
        m = O.uniform(40 + b, 1, t, n)
        msgs.append(m)
        cts.append(lat.encrypt(k, sk_ntt, base.wrapping_decompose_small(m, t), lat.delta(t), 9 + b))
    table = gpu.DcrtTable(log_n, moduli)
    dec = gpu.BfvDecryptor(table, t, gamma)
    out = gpu.DeviceBuffer(batch * n)
    dec.decrypt(k, gpu.DeviceBuffer.from_numpy(sk_ntt), gpu.DeviceBuffer.from_numpy(np.concatenate(cts)), out, batch)
    got = out.numpy().reshape(batch, n)
    for b in range(batch):
        assert np.array_equal(got[b], lat.decrypt(k, sk_ntt, cts[b], t, gamma))
        assert np.array_equal(got[b], msgs[b])


def test_decryptor_rejects_non_coprime(gpu):
    moduli = O.ntt_primes(1 << 50, 2048, 2)
    table = gpu.DcrtTable(10, moduli)
    with pytest.raises(gpu.PrimusGpuError):
        gpu.BfvDecryptor(table, 16, 256)  # gamma even, t even
    with pytest.raises(gpu.PrimusGpuError):
        gpu.BfvDecryptor(table, 17, int(moduli[0]))  # gamma equal to a modulus
