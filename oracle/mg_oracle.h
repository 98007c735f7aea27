/*
 * mg_oracle.h -- CPU oracle for the per-server ChaCha8-DPF PIR answer path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * CPU algorithm (crates/morphogen-gpu-dpf/src/{chacha_prg,dpf,kernel}.rs and
 * crates/morphogen-server/src/scan.rs), used as the checker by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline / reference arm.  The
 * product library never links, loads or calls it.
 *
 * Parity pins (see tests/test_oracle.py):
 *   - the ChaCha core, run with 10 double rounds, equals OpenSSL's ChaCha20
 *     keystream (Python `cryptography`), fixtures in tests/golden/;
 *   - the DPF properties the reference's own tests assert (dpf.rs:474-584,
 *     kernel.rs:1444-1561): share XOR = point function / target row;
 *   - page-mode shares equal those of the reference's own CUDA kernels built
 *     from the reference sources into oracle/_ref (GPU test).
 *
 * Rows generalise the reference's 4096-B pages: a row is R bytes, R % 16 == 0,
 * and the 16-byte DPF output is repeated over each 16-byte lane of the row
 * (the convention of kernel.rs:1243-1256 and scan.rs:478-480).
 */
#ifndef MG_ORACLE_H
#define MG_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MGO_MAX_LEVELS 64

typedef struct {
  uint32_t root_seed[4];
  uint8_t root_t;  /* byte, as in the reference (dpf.rs:94) */
  uint8_t party;
  uint32_t domain_bits;
  uint32_t cw_seed[MGO_MAX_LEVELS][4];
  uint8_t cw_tl[MGO_MAX_LEVELS];
  uint8_t cw_tr[MGO_MAX_LEVELS];
  uint32_t final_cw[4];
} mgo_key;

/* chacha_prg.rs:112-144 with a configurable number of double rounds
 * (4 = ChaCha8 as in the reference; 10 = ChaCha20, used only for pinning). */
void mgo_chacha_block(const uint32_t key[8], uint32_t counter, const uint32_t nonce[3],
                      int double_rounds, uint32_t out[16]);

/* chacha_prg.rs:153-178. */
void mgo_prg_expand(const uint32_t seed[4], uint32_t left[4], uint32_t right[4],
                    uint8_t* left_t, uint8_t* right_t);

/* dpf.rs:277-316 (returns 0 or -1 for a malformed length). */
int mgo_key_from_bytes(const uint8_t* bytes, size_t len, mgo_key* key);
/* dpf.rs:259-274 (returns bytes written: 19 + 18 d + 16). */
size_t mgo_key_to_bytes(const mgo_key* key, uint8_t* out);

/* dpf.rs:103-142. */
void mgo_eval(const mgo_key* key, uint64_t index, uint32_t out[4]);
/* dpf.rs:164-246: aligned subtree of n (power of two) leaves at start. */
int mgo_eval_subtree(const mgo_key* key, uint64_t start, uint64_t n, uint32_t* out /* n*4 */);

/* dpf.rs:322-432 with the two root seeds supplied by the caller (the
 * reference draws them from an unseeded rand::random). */
int mgo_keygen(uint32_t domain_bits, uint64_t target, const uint32_t seed0[4],
               const uint32_t seed1[4], mgo_key* k0, mgo_key* k1);

/* kernel.rs:1276-1371 generalised to nkeys keys and R-byte rows.  rows holds
 * nrows rows whose DPF indices are row_base .. row_base + nrows - 1; out is
 * nkeys * row_bytes.  Tiles of min(2048, 2^d) leaves, OpenMP over tiles with
 * nthreads threads (<= 0: all).  Returns 0, or -1 on a precondition error. */
int mgo_scan_fused(const mgo_key* keys, int nkeys, const uint8_t* rows, uint64_t nrows,
                   uint32_t row_bytes, uint64_t row_base, uint8_t* out, int nthreads);

/* kernel.rs:1374-1383: one key, one point evaluation per row. */
/* mgo_scan_fused with the AND/XOR loop in AVX-512 registers, eight rows per
 * step (the shape of crates/morphogen-server/src/scan.rs:719-895); scalar
 * ChaCha8 as the reference's CPU path.  Same result; -2 without AVX-512F. */
int mgo_scan_fused_avx512(const mgo_key* keys, int nkeys, const uint8_t* rows, uint64_t nrows,
                          uint32_t row_bytes, uint64_t row_base, uint8_t* out, int nthreads);
int mgo_avx512_available(void);

int mgo_scan_pointwise(const mgo_key* key, const uint8_t* rows, uint64_t nrows,
                       uint32_t row_bytes, uint8_t* out);

/* scan.rs:434-485 in row mode: for each delta entry and key,
 * out[k] ^= diff & eval(row_idx) (mask repeated per 16-byte lane). */
int mgo_delta_apply(const mgo_key* keys, int nkeys, const uint64_t* row_idx,
                    const uint8_t* diffs, uint64_t nentries, uint32_t row_bytes, uint8_t* out);

/* Counter-based table generator: byte o = byte (o % 8) of
 * splitmix64_output(seed, o / 8).  Any byte range can be regenerated. */
void mgo_fill_splitmix(uint8_t* buf, uint64_t byte_offset, uint64_t nbytes, uint64_t seed);
uint64_t mgo_splitmix_word(uint64_t seed, uint64_t index);

/* morphogen-storage/src/chunked_matrix.rs:83-93 (sequential LCG). */
void mgo_fill_lcg(uint8_t* buf, uint64_t nbytes, uint64_t seed);

/* kernel.rs:1390-1403 (make_test_pages), generalised to R-byte rows. */
void mgo_fill_test_rows(uint8_t* buf, uint64_t nrows, uint32_t row_bytes);

#ifdef __cplusplus
}
#endif
#endif
