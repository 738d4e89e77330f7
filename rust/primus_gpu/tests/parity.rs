//! Parity of the GPU tables with the reference's CPU tables on the same inputs
//! (needs a CUDA device).  Mirrors primus_ntt/tests/hexl.rs: every transform of
//! the GPU table equals UintNttTable's, lazy values included.
use primus_gpu::{GpuDcrtTable, GpuNttTable};
use primus_modulus::BarrettModulus;
use primus_ntt::{DcrtTable, NttTable, UintCrtNttTable, UintNttTable};
use primus_reduce::Modulus;

fn seeded(n: usize, q: u64, seed: u64) -> Vec<u64> {
    // splitmix64: any fixed sequence of residues will do
    let mut s = seed;
    (0..n)
        .map(|_| {
            s = s.wrapping_add(0x9E3779B97F4A7C15);
            let mut z = s;
            z = (z ^ (z >> 30)).wrapping_mul(0xBF58476D1CE4E5B9);
            z = (z ^ (z >> 27)).wrapping_mul(0x94D049BB133111EB);
            (z ^ (z >> 31)) % q
        })
        .collect()
}

#[test]
fn ntt_table_matches_uint_table() {
    let q: u64 = 1125899906826241; // the largest prime below 2^50 with q = 1 mod 2^13
    for log_n in [4u32, 10] {
        let m = BarrettModulus::<u64>::new(q);
        let cpu = UintNttTable::<u64>::new(log_n, m).unwrap();
        let gpu = GpuNttTable::new(log_n, m).unwrap();
        let a = seeded(1 << log_n, q, log_n as u64);
        let (mut x, mut y) = (a.clone(), a.clone());
        cpu.lazy_transform_slice(&mut x);
        gpu.lazy_transform_slice(&mut y);
        assert_eq!(x, y);
        cpu.inverse_transform_slice(&mut x);
        gpu.inverse_transform_slice(&mut y);
        assert_eq!(x, y);
        assert_eq!(x, a);
    }
}

#[test]
fn dcrt_table_matches_uint_crt_table() {
    let moduli: Vec<BarrettModulus<u64>> =
        [1125899906826241u64, 1125899906629633].iter().map(|&q| BarrettModulus::new(q)).collect();
    let log_n = 12;
    let cpu = UintCrtNttTable::<u64>::new(log_n, &moduli).unwrap();
    let gpu = GpuDcrtTable::new(log_n, &moduli).unwrap();
    let mut a = seeded(1 << log_n, moduli[0].value_unchecked(), 1);
    a.extend(seeded(1 << log_n, moduli[1].value_unchecked(), 2));
    let (mut x, mut y) = (a.clone(), a.clone());
    cpu.transform_slice(&mut x);
    gpu.transform_slice(&mut y);
    assert_eq!(x, y);
    for (t, c) in gpu.iter().zip(cpu.iter()) {
        let (mut m1, mut m2) = (vec![0u64; 1 << log_n], vec![0u64; 1 << log_n]);
        t.transform_monomial(3, 5, &mut m1);
        c.transform_monomial(3, 5, &mut m2);
        assert_eq!(m1, m2);
    }
}
