"""CPU check of the bench's own output verification (bench.RowCheck).

The bench regenerates four rows (one limb each of four polys) from the seed and
carries them through the same round trips with the oracle.  Here the rows it
predicts after two round trips are compared with the same rows taken out of
whole-poly oracle round trips of those polys (UintCrtNttTable transforms and the
pointwise product with the NTT-domain plaintext), so that a wrong seed, stream,
limb or plaintext index in RowCheck cannot make the bench report "verified"."""
import bench
import oracle as O


def test_rowcheck_rows_follow_whole_poly_round_trips():
    moduli = O.ntt_primes(1 << 50, 2 * bench.N, bench.L)
    seed = bench.SEED + 1  # a replica rank's seed, as the bench uses SEED + rank
    rc = bench.RowCheck(moduli, seed, threads=8)
    full = O.DcrtTable(bench.LOG_N, moduli)
    plain = full.forward(O.uniform_rns(bench.SEED + 7, 0, moduli, bench.N), threads=8)
    rows, rows1 = {}, {}
    for p in rc.polys:
        x = O.uniform_rns(seed, p * bench.L, moduli, bench.N)
        for k in range(2):
            x = full.polymul_roundtrip(x, plain, threads=8).reshape(x.shape)
            if k == 0:
                rows1[p] = x.reshape(bench.L, bench.N).copy()
        rows[p] = x.reshape(bench.L, bench.N)

    def read(row):
        return rows[row // bench.L][row % bench.L]

    assert rc.check("two round trips", 2, read)
    # a later leg may have run fewer round trips on its own copy of the batch
    assert rc.check("one round trip", 1, lambda row: rows1[row // bench.L][row % bench.L])
    assert rc.check("two round trips again", 2, read)
    assert rc.summary()["verified"]
    # rows one limb off do not pass, nor rows one round trip off
    assert not rc.check("rows one limb off", 2, lambda row: rows[row // bench.L][(row + 1) % bench.L])
    assert not rc.check("rows one round trip off", 1, read)
    assert not rc.summary()["verified"]
