"""numpy restatement of the reference client library's wire formats.

Test infrastructure only, like the rest of oracle/: the tests and the
golden-fixture generator use it to check the server's packed and compressed
outputs; the product never imports it.

* 53-bit packed query / response: each coefficient's two residues are
  combined by CRT (Garner, src/capi_client.cpp:160-179) into one value below
  q0*q1 < 2^53, written MSB first at 53 bits per value with the last byte
  zero-padded (BitWriter / BitReader, src/capi_client.cpp:184-222).  Query
  order: the R LWE coefficients, then the 6*d_eff key/RGSW polynomials
  coefficient by coefficient (src/capi_client.cpp:246-277); response order:
  a then b of each ciphertext (src/capi_client.cpp:279-289).  Unpacking
  reduces each value mod q0 and mod q1.
* Compressed response (src/capi_client.cpp:355-385, src/crypto.cpp:285-313):
  per ciphertext, a and b to coefficient form (inverse NTT), each
  coefficient lifted to [0, Q), Q = q0*q1, rounded to q' = 2^28 (a) or 2^20
  (b) as floor((v q' + floor(Q/2)) / Q) mod q', then N x 28 bits of a and
  N x 20 bits of b, MSB first, the ciphertext's last byte zero-padded
  (12288 bytes per ciphertext, no padding at N = 2048).
"""
import numpy as np

N = 2048
Q0, Q1 = 94519297, 95293441
D_EFF = 2
WIRE_BITS = 53
MASK_BITS, BODY_BITS = 28, 20
Q_FULL = Q0 * Q1
Q1_INV_Q0 = pow(Q1, -1, Q0)
Q0_INV_Q1 = pow(Q0, -1, Q1)


def _pack_bits(values, bits):
    """values (u64, each < 2^bits) -> bytes, MSB first, last byte zero-padded."""
    v = np.ascontiguousarray(values, np.uint64)
    shifts = np.arange(bits - 1, -1, -1, dtype=np.uint64)
    b = ((v[:, None] >> shifts[None, :]) & np.uint64(1)).astype(np.uint8)
    return np.packbits(b.reshape(-1))


def _unpack_bits(data, count, bits):
    """First count values of `bits` bits each from MSB-first bytes."""
    b = np.unpackbits(np.ascontiguousarray(data, np.uint8))[: count * bits]
    if b.size != count * bits:
        raise ValueError("packed stream too short")
    shifts = np.arange(bits - 1, -1, -1, dtype=np.uint64)
    return (b.reshape(count, bits).astype(np.uint64) << shifts[None, :]).sum(axis=1, dtype=np.uint64)


def crt_combine(v0, v1):
    """Garner: v1 + q1 ((v0 - v1) q1^-1 mod q0), for v0 < q0, v1 < q1 (u64 arrays)."""
    v0 = np.asarray(v0, np.uint64)
    v1 = np.asarray(v1, np.uint64)
    diff = (v0 + np.uint64(Q0) - v1 % np.uint64(Q0)) % np.uint64(Q0)
    h = (diff * np.uint64(Q1_INV_Q0)) % np.uint64(Q0)   # < 2^27 * 2^27: no overflow
    return v1 + np.uint64(Q1) * h


def query_values(rows):
    return rows + 6 * D_EFF * N


def query_packed_bytes(rows):
    return (query_values(rows) * WIRE_BITS + 7) // 8


def response_packed_bytes(num_cts):
    return (num_cts * 2 * N * WIRE_BITS + 7) // 8


def compressed_bytes(num_cts):
    return num_cts * N * (MASK_BITS + BODY_BITS) // 8


def pack_query(flat, rows):
    """Flat u64 query [lwe0 R][lwe1 R][12 polys x (limb0 N, limb1 N)] -> packed bytes."""
    flat = np.ascontiguousarray(flat, np.uint64)
    polys = flat[2 * rows:].reshape(6 * D_EFF, 2, N)
    v = np.concatenate([crt_combine(flat[:rows], flat[rows:2 * rows]),
                        crt_combine(polys[:, 0, :], polys[:, 1, :]).reshape(-1)])
    return _pack_bits(v, WIRE_BITS)


def unpack_query(data, rows):
    v = _unpack_bits(data, query_values(rows), WIRE_BITS)
    out = np.empty(2 * rows + 6 * D_EFF * 2 * N, np.uint64)
    out[:rows] = v[:rows] % np.uint64(Q0)
    out[rows:2 * rows] = v[:rows] % np.uint64(Q1)
    pv = v[rows:].reshape(6 * D_EFF, N)
    polys = out[2 * rows:].reshape(6 * D_EFF, 2, N)
    polys[:, 0, :] = pv % np.uint64(Q0)
    polys[:, 1, :] = pv % np.uint64(Q1)
    return out


def pack_response(flat, num_cts):
    """Flat u64 response [ct][a|b][limb][N] -> packed bytes."""
    p = np.ascontiguousarray(flat, np.uint64).reshape(num_cts * 2, 2, N)
    return _pack_bits(crt_combine(p[:, 0, :], p[:, 1, :]).reshape(-1), WIRE_BITS)


def unpack_response(data, num_cts):
    v = _unpack_bits(data, num_cts * 2 * N, WIRE_BITS).reshape(num_cts * 2, N)
    out = np.empty((num_cts * 2, 2, N), np.uint64)
    out[:, 0, :] = v % np.uint64(Q0)
    out[:, 1, :] = v % np.uint64(Q1)
    return out.reshape(-1)


def _mod_switch(c0, c1, bits):
    """Exact lift to [0, Q) and rounding to 2^bits, in Python integers."""
    out = np.empty(len(c0), np.uint64)
    half = Q_FULL // 2
    for i, (x0, x1) in enumerate(zip(c0.tolist(), c1.tolist())):
        v = ((x0 * Q1_INV_Q0 % Q0) * Q1 + (x1 * Q0_INV_Q1 % Q1) * Q0) % Q_FULL
        out[i] = ((v << bits) + half) // Q_FULL % (1 << bits)
    return out


def compress_response(flat, num_cts, ntt_inverse):
    """Flat NTT-form response -> compressed bytes.  ntt_inverse(poly, limb)
    is the negacyclic inverse NTT of one limb (the oracle's)."""
    p = np.ascontiguousarray(flat, np.uint64).reshape(num_cts, 2, 2, N)
    parts = []
    for ct in range(num_cts):
        coef = [[ntt_inverse(p[ct, ab, l], l) for l in (0, 1)] for ab in (0, 1)]
        a = _mod_switch(coef[0][0], coef[0][1], MASK_BITS)
        b = _mod_switch(coef[1][0], coef[1][1], BODY_BITS)
        parts.append(np.packbits(np.concatenate([
            ((a[:, None] >> np.arange(MASK_BITS - 1, -1, -1, dtype=np.uint64)) & np.uint64(1)).reshape(-1),
            ((b[:, None] >> np.arange(BODY_BITS - 1, -1, -1, dtype=np.uint64)) & np.uint64(1)).reshape(-1),
        ]).astype(np.uint8)))
    return np.concatenate(parts)


def splitmix_db(count, seed):
    """The parity cases' synthetic DB: splitmix64(seed ^ k) mod 65535 at flat index k."""
    k = np.arange(count, dtype=np.uint64)
    with np.errstate(over="ignore"):
        x = (k ^ np.uint64(seed)) + np.uint64(0x9E3779B97F4A7C15)
        x = (x ^ (x >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        x = (x ^ (x >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        x ^= x >> np.uint64(31)
    return (x % np.uint64(65535)).astype(np.uint16)
