//! Keys with the reference's types and wire format
//! (crates/morphogen-gpu-dpf/src/dpf.rs, chacha_prg.rs:14-74).  Parsing and
//! serialisation are plain Rust; key generation runs in the library
//! (mg_keygen, the restated generate_chacha_dpf_keys of dpf.rs:322-432) with
//! root seeds from the operating system's random source, as the reference
//! draws them from rand::random (chacha_prg.rs:67-72).
use std::convert::TryInto;

use crate::ffi;

/// 128-bit seed for DPF nodes: four little-endian words (chacha_prg.rs:14-74).
#[derive(Clone, Copy, Debug, PartialEq, Eq, Default)]
#[repr(C)]
pub struct Seed128 {
    pub words: [u32; 4],
}

impl Seed128 {
    pub const ZERO: Self = Self { words: [0; 4] };

    pub fn new(words: [u32; 4]) -> Self {
        Self { words }
    }

    pub fn from_bytes(bytes: &[u8; 16]) -> Self {
        let mut words = [0u32; 4];
        for (i, w) in words.iter_mut().enumerate() {
            *w = u32::from_le_bytes(bytes[4 * i..4 * i + 4].try_into().unwrap());
        }
        Self { words }
    }

    pub fn to_bytes(&self) -> [u8; 16] {
        let mut out = [0u8; 16];
        for (i, w) in self.words.iter().enumerate() {
            out[4 * i..4 * i + 4].copy_from_slice(&w.to_le_bytes());
        }
        out
    }

    pub fn xor(&self, other: &Self) -> Self {
        let mut words = self.words;
        for (w, o) in words.iter_mut().zip(other.words.iter()) {
            *w ^= *o;
        }
        Self { words }
    }

    pub fn and(&self, other: &Self) -> Self {
        let mut words = self.words;
        for (w, o) in words.iter_mut().zip(other.words.iter()) {
            *w &= *o;
        }
        Self { words }
    }

    /// A seed from the operating system's random source.
    pub fn random() -> Self {
        Self::from_bytes(&os_random_16())
    }
}

fn os_random_16() -> [u8; 16] {
    use std::io::Read;
    let mut b = [0u8; 16];
    std::fs::File::open("/dev/urandom")
        .and_then(|mut f| f.read_exact(&mut b))
        .expect("reading /dev/urandom");
    b
}

/// dpf.rs:9-15, with the same messages.
#[derive(Debug, Clone)]
pub enum GpuDpfError {
    InvalidDomainBits { bits: usize, reason: &'static str },
    PageIndexTooLarge { index: usize, max: usize },
    InvalidKeyLength { expected: usize, actual: usize },
    InvalidKeyFormat(&'static str),
}

impl std::fmt::Display for GpuDpfError {
    fn fmt(&self, f: &mut std::fmt::Formatter<'_>) -> std::fmt::Result {
        match self {
            Self::InvalidDomainBits { bits, reason } => write!(f, "Invalid domain bits {}: {}", bits, reason),
            Self::PageIndexTooLarge { index, max } => write!(f, "Page index {} exceeds max {}", index, max),
            Self::InvalidKeyLength { expected, actual } => {
                write!(f, "Invalid key length: expected {}, got {}", expected, actual)
            }
            Self::InvalidKeyFormat(reason) => write!(f, "Invalid key format: {}", reason),
        }
    }
}

impl std::error::Error for GpuDpfError {}

/// Correction word of one tree level (dpf.rs:43-56).
#[derive(Clone, Copy, Debug)]
pub struct CorrectionWord {
    pub seed_cw: Seed128,
    pub t_cw_left: u8,
    pub t_cw_right: u8,
}

impl CorrectionWord {
    pub const ZERO: Self = Self { seed_cw: Seed128::ZERO, t_cw_left: 0, t_cw_right: 0 };
}

/// dpf.rs:59-86.
#[derive(Clone, Debug)]
pub struct ChaChaParams {
    pub domain_bits: usize,
}

impl ChaChaParams {
    pub fn new(domain_bits: usize) -> Result<Self, GpuDpfError> {
        if domain_bits == 0 {
            return Err(GpuDpfError::InvalidDomainBits { bits: domain_bits, reason: "must be > 0" });
        }
        if domain_bits > 32 {
            return Err(GpuDpfError::InvalidDomainBits { bits: domain_bits, reason: "must be <= 32" });
        }
        Ok(Self { domain_bits })
    }

    pub fn max_pages(&self) -> usize {
        1usize.checked_shl(self.domain_bits as u32).unwrap_or(usize::MAX)
    }
}

/// One party's DPF key (dpf.rs:92-99).  Domains up to 32 levels are
/// evaluated in full on the device (the reference kernel stops at 25).
#[derive(Clone, Debug)]
pub struct ChaChaKey {
    pub root_seed: Seed128,
    pub root_t: u8,
    pub domain_bits: usize,
    pub correction_words: Vec<CorrectionWord>,
    pub final_cw: Seed128,
    pub party: u8,
}

impl ChaChaKey {
    pub fn max_pages(&self) -> usize {
        1usize.checked_shl(self.domain_bits as u32).unwrap_or(usize::MAX)
    }

    pub fn is_party1(&self) -> bool {
        self.party == 1
    }

    /// Wire format of dpf.rs:259-274: seed, root t, party, depth, per level
    /// (seed CW, tL, tR), final CW.
    pub fn to_bytes(&self) -> Vec<u8> {
        let mut bytes = Vec::with_capacity(35 + self.correction_words.len() * 18);
        bytes.extend_from_slice(&self.root_seed.to_bytes());
        bytes.push(self.root_t);
        bytes.push(self.party);
        bytes.push(self.domain_bits as u8);
        for cw in &self.correction_words {
            bytes.extend_from_slice(&cw.seed_cw.to_bytes());
            bytes.push(cw.t_cw_left);
            bytes.push(cw.t_cw_right);
        }
        bytes.extend_from_slice(&self.final_cw.to_bytes());
        bytes
    }

    /// dpf.rs:277-316, same checks and messages.
    pub fn from_bytes(bytes: &[u8]) -> Result<Self, GpuDpfError> {
        if bytes.len() < 19 + 16 {
            return Err(GpuDpfError::InvalidKeyFormat("Byte array too short"));
        }
        let domain_bits = bytes[18] as usize;
        if bytes.len() != 19 + domain_bits * 18 + 16 {
            return Err(GpuDpfError::InvalidKeyFormat("Invalid byte array length"));
        }
        let seed = |off: usize| Seed128::from_bytes(bytes[off..off + 16].try_into().unwrap());
        let correction_words = (0..domain_bits)
            .map(|l| {
                let off = 19 + 18 * l;
                CorrectionWord { seed_cw: seed(off), t_cw_left: bytes[off + 16], t_cw_right: bytes[off + 17] }
            })
            .collect();
        Ok(Self {
            root_seed: seed(0),
            root_t: bytes[16],
            party: bytes[17],
            domain_bits,
            correction_words,
            final_cw: seed(19 + 18 * domain_bits),
        })
    }
}

/// dpf.rs:322-432: the two parties' keys for `target` (their evaluations
/// XOR to all-ones at the target and to zero elsewhere).
pub fn generate_chacha_dpf_keys(params: &ChaChaParams, target: usize) -> Result<(ChaChaKey, ChaChaKey), GpuDpfError> {
    let max = params.max_pages();
    if target >= max {
        return Err(GpuDpfError::PageIndexTooLarge { index: target, max });
    }
    generate_chacha_dpf_keys_with_seeds(params, target, Seed128::random(), Seed128::random())
}

/// generate_chacha_dpf_keys with caller-chosen root seeds (seeded runs).
pub fn generate_chacha_dpf_keys_with_seeds(params: &ChaChaParams, target: usize, seed0: Seed128, seed1: Seed128)
    -> Result<(ChaChaKey, ChaChaKey), GpuDpfError> {
    let max = params.max_pages();
    if target >= max {
        return Err(GpuDpfError::PageIndexTooLarge { index: target, max });
    }
    let d = params.domain_bits as u32;
    let n = unsafe { ffi::mg_key_size(d) };
    let mut k0 = vec![0u8; n];
    let mut k1 = vec![0u8; n];
    let (r0, r1) = (seed0.to_bytes(), seed1.to_bytes());
    let rc = unsafe { ffi::mg_keygen(d, target as u64, r0.as_ptr(), r1.as_ptr(), k0.as_mut_ptr(), k1.as_mut_ptr()) };
    if rc != ffi::MG_OK {
        return Err(GpuDpfError::InvalidKeyFormat("key generation rejected the parameters"));
    }
    Ok((ChaChaKey::from_bytes(&k0)?, ChaChaKey::from_bytes(&k1)?))
}

#[cfg(test)]
mod tests {
    use super::*;

    #[test]
    fn serialization_roundtrip() {
        let key = ChaChaKey {
            root_seed: Seed128::new([1, 2, 3, 4]),
            root_t: 1,
            domain_bits: 3,
            correction_words: vec![CorrectionWord { seed_cw: Seed128::new([5, 6, 7, 8]), t_cw_left: 1, t_cw_right: 0 }; 3],
            final_cw: Seed128::new([9, 10, 11, 12]),
            party: 1,
        };
        let b = key.to_bytes();
        assert_eq!(b.len(), 19 + 3 * 18 + 16);
        let back = ChaChaKey::from_bytes(&b).unwrap();
        assert_eq!(back.to_bytes(), b);
        assert!(back.is_party1());
        assert!(ChaChaKey::from_bytes(&b[..20]).is_err());
    }

    #[test]
    fn params_bounds() {
        assert!(ChaChaParams::new(0).is_err());
        assert!(ChaChaParams::new(33).is_err());
        assert_eq!(ChaChaParams::new(31).unwrap().max_pages(), 1 << 31);
    }
}
