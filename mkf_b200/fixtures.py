"""Fixture directories of the reference's bit-exact exporters: read them, run
them through the GPU path, and write our own in the same format.

The reference exports opt-in fixtures for its FPGA harness
(software/mkf/mkf_cpu/fpga_fixture_test.go:24-129, 280-390 for MKF-CKKS and
MKF-BFV; software/kklss/mkckks/fpga_fixture_test.go:22-248 for KKLSS-CKKS):
a `manifest.json` (moduli, degree, parties, levels, beta, file names,
SHA-256 of every file) beside little-endian uint64 files, modulus-major then
coefficient-major -- exactly the library's limb-major layout, so every file
maps onto a C-ABI buffer without conversion:

* MKF: `input_ciphertexts_q.bin` = side[left,right], component[c0, party0..],
  `fold_and_relin_keys_qp.bin` = fold key per party then the aggregate relin
  key, each [beta][2][Q then P], `expected_output_q.bin` = c0, gamma, then
  gamma repeated per party (the paper's (n+1)-component interface); optional
  stage dumps (`debug_switch0_*.bin`, `stage_fold_q.bin`).
* KKLSS: `input_ciphertexts_q.bin` = side[left,right], component in
  `ciphertext_order`, `relinearization_keys_qp.bin` = per user (b, d, v) each
  [beta][Q then P], `crs_u_qp.bin` = [beta][Q then P],
  `expected_ciphertext_q.bin` = components in `ciphertext_order`.

`load` + `run` diff a fixture (for instance one exported by the Go reference
on a machine with Lattigo v2.3.0) against the GPU path; `export_mkf` /
`export_kklss` write fixtures from any source (the tests use the oracle), and
the key files double as a persistence format for key pools.
"""
from __future__ import annotations

import hashlib
import json
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import params
from .params import ParametersLiteral

MKF_FILES = {"inputs": "input_ciphertexts_q.bin", "keys": "fold_and_relin_keys_qp.bin",
             "output": "expected_output_q.bin"}
KKLSS_FILES = {"inputs": "input_ciphertexts_q.bin", "keys": "relinearization_keys_qp.bin",
               "crs": "crs_u_qp.bin", "output": "expected_ciphertext_q.bin"}


def sha256_file(path: str) -> str:
    h = hashlib.sha256()
    with open(path, "rb") as f:
        for chunk in iter(lambda: f.read(1 << 22), b""):
            h.update(chunk)
    return h.hexdigest()


def _read_words(path: str, count: Optional[int] = None) -> np.ndarray:
    a = np.fromfile(path, dtype="<u8")
    if count is not None and a.size != count:
        raise ValueError(f"{os.path.basename(path)}: {a.size} words, expected {count}")
    return a.astype(np.uint64, copy=False)


def _write_words(path: str, *arrays: np.ndarray):
    with open(path, "wb") as f:
        for a in arrays:
            np.ascontiguousarray(a, dtype="<u8").tofile(f)


@dataclass
class Fixture:
    dir: str
    manifest: dict
    scheme: str          # "MKF-CKKS", "MKF-BFV", "KKLSS-CKKS" or "KKLSS-BFV"
    lit: ParametersLiteral
    k: int
    level_in: int
    level_out: int
    beta: int
    left: np.ndarray     # [k+1][level_in+1][N]
    right: np.ndarray
    expected: np.ndarray  # [components][level_out+1][N]
    fold: Optional[np.ndarray] = None   # MKF: [k][beta][2][nQ+nP][N]
    relin: Optional[np.ndarray] = None  # MKF: [beta][2][nQ+nP][N]
    rlk: Dict[int, np.ndarray] = field(default_factory=dict)  # KKLSS: party -> key words
    crs_u: Optional[np.ndarray] = None
    ids: List[int] = field(default_factory=list)

    @property
    def is_ckks(self) -> bool:
        return self.scheme.endswith("CKKS")


def read_manifest(d: str) -> dict:
    with open(os.path.join(d, "manifest.json")) as f:
        return json.load(f)


def verify_hashes(d: str, manifest: dict) -> List[str]:
    """Files whose SHA-256 differs from the manifest's."""
    bad = []
    for name, want in (manifest.get("sha256") or {}).items():
        p = os.path.join(d, name)
        if not os.path.exists(p) or sha256_file(p) != want:
            bad.append(name)
    return bad


def literal_from_manifest(m: dict) -> ParametersLiteral:
    """Parameter literal of a fixture.  CKKS scale: the named set's when its
    moduli match (P1, P2, C1, C3, S14-S16), else the last modulus at the input
    level (one rescale, as every CKKS fixture of the reference performs)."""
    n = int(m["polynomial_degree"])
    log_n = n.bit_length() - 1
    if 1 << log_n != n:
        raise ValueError("polynomial_degree is not a power of two")
    q, p = tuple(int(x) for x in m["q"]), tuple(int(x) for x in m["p"])
    qm = tuple(int(x) for x in (m.get("q_mul") or ()))
    ckks = m["scheme"].endswith("CKKS")
    named = None
    try:
        named = params.get("ckks" if ckks else "bfv", m.get("parameter", ""))
    except ValueError:
        pass
    if named is not None and named.q == q and named.p == p and (ckks or named.q_mul == qm):
        return named
    if ckks:
        scale = float(q[int(m["input_level_q"])])
        return ParametersLiteral(m.get("parameter", "fixture"), log_n, q, p, (), log_n - 1, scale)
    return ParametersLiteral(m.get("parameter", "fixture"), log_n, q, p, qm,
                             t=int(m.get("plaintext_modulus", 0)))


def load(d: str, check_hashes: bool = True) -> Fixture:
    m = read_manifest(d)
    if check_hashes:
        bad = verify_hashes(d, m)
        if bad:
            raise ValueError(f"SHA-256 mismatch for {bad}")
    lit = literal_from_manifest(m)
    scheme = m["scheme"]
    N, nQ, nP = lit.n, len(lit.q), len(lit.p)
    k = int(m["parties"])
    li, lo, beta = int(m["input_level_q"]), int(m["output_level_q"]), int(m["beta"])
    L1 = li + 1
    qp = (nQ + nP) * N
    ins = _read_words(os.path.join(d, m.get("input_file") or m.get("input_ciphertexts_file")),
                      2 * (k + 1) * L1 * N).reshape(2, k + 1, L1, N)
    # keys hold every decomposition of the top level; the manifest's beta is
    # the input level's, so the key shape comes from the file size
    if scheme.startswith("MKF"):
        keys = _read_words(os.path.join(d, m["switching_key_file"]))
        kb = keys.size // ((k + 1) * 2 * qp)
        if kb * (k + 1) * 2 * qp != keys.size:
            raise ValueError("switching-key file size is not (k+1) whole keys")
        keys = keys.reshape(k + 1, kb, 2, nQ + nP, N)
        out = _read_words(os.path.join(d, m["output_file"]), (k + 2) * (lo + 1) * N)
        return Fixture(d, m, scheme, lit, k, li, lo, beta, ins[0], ins[1],
                       out.reshape(k + 2, lo + 1, N), fold=keys[:k], relin=keys[k])
    order = list(m["ciphertext_order"])
    crs = _read_words(os.path.join(d, m["crs_u_file"]))
    kb = crs.size // qp
    if kb * qp != crs.size:
        raise ValueError("CRS file size is not whole decompositions")
    per = (3 if scheme == "KKLSS-CKKS" else 6) * kb * qp
    keys = _read_words(os.path.join(d, m["relinearization_key_file"]), k * per).reshape(k, per)
    out = _read_words(os.path.join(d, m["output_ciphertext_file"]), (k + 1) * (lo + 1) * N)
    ids = list(range(k))
    if len(order) != k + 1 or order[0] != "0":
        raise ValueError("ciphertext_order must be component 0 then one entry per party")
    return Fixture(d, m, scheme, lit, k, li, lo, beta, ins[0], ins[1], out.reshape(k + 1, lo + 1, N),
                   rlk={i: keys[i] for i in ids}, crs_u=crs, ids=ids)


def _manifest(scheme, parameter, lit, k, li, lo, beta, files, orders) -> dict:
    m = {"scheme": scheme, "parameter": parameter, "parties": k, "polynomial_degree": lit.n,
         "q": [int(x) for x in lit.q], "p": [int(x) for x in lit.p],
         "input_level_q": li, "output_level_q": lo, "beta": beta}
    if lit.q_mul:
        m["q_mul"] = [int(x) for x in lit.q_mul]
    if lit.t:
        m["plaintext_modulus"] = int(lit.t)
    m.update(orders)
    m.update(files)
    return m


def _finish(d: str, m: dict, names):
    m["sha256"] = {n: sha256_file(os.path.join(d, n)) for n in names}
    with open(os.path.join(d, "manifest.json"), "w") as f:
        f.write(json.dumps(m, indent=2) + "\n")


def export_mkf(d: str, scheme: str, parameter: str, lit: ParametersLiteral, left, right, fold, relin,
               output, level_out: int) -> dict:
    """Writes an MKF fixture.  output: the compact (c0, gamma) pair or the
    materialized c0 + k gammas; the file holds c0, gamma, gamma x k."""
    os.makedirs(d, exist_ok=True)
    left, right = np.asarray(left, np.uint64), np.asarray(right, np.uint64)
    k = left.shape[0] - 1
    li = left.shape[1] - 1
    beta = np.asarray(relin).shape[0]
    out = np.asarray(output, np.uint64)
    gamma = out[1]
    _write_words(os.path.join(d, MKF_FILES["inputs"]), left, right)
    _write_words(os.path.join(d, MKF_FILES["keys"]), *[np.asarray(f, np.uint64) for f in fold],
                 np.asarray(relin, np.uint64))
    _write_words(os.path.join(d, MKF_FILES["output"]), out[0], gamma, *([gamma] * k))
    m = _manifest(scheme, parameter, lit, k, li, level_out, beta,
                  {"input_file": MKF_FILES["inputs"], "switching_key_file": MKF_FILES["keys"],
                   "output_file": MKF_FILES["output"]},
                  {"input_order": "side[left,right], component[c0,party0..], modulus, coefficient",
                   "switching_key_order": "fold_key[party0..], then aggregate_relin_key; decomposition, "
                                          "output_poly[0..1], Q_then_P, modulus, coefficient",
                   "output_order": "c0, gamma, repeated_gamma[party0..], modulus, coefficient"})
    _finish(d, m, MKF_FILES.values())
    return m


def export_kklss(d: str, scheme: str, parameter: str, lit: ParametersLiteral, left, right,
                 rlk: List[np.ndarray], crs_u, output, level_out: int) -> dict:
    """Writes a KKLSS fixture; parties are user0..user{k-1} in component order."""
    os.makedirs(d, exist_ok=True)
    left, right = np.asarray(left, np.uint64), np.asarray(right, np.uint64)
    k = left.shape[0] - 1
    li = left.shape[1] - 1
    N, nQ, nP = lit.n, len(lit.q), len(lit.p)
    beta = np.asarray(crs_u).size // ((nQ + nP) * N)
    _write_words(os.path.join(d, KKLSS_FILES["inputs"]), left, right)
    _write_words(os.path.join(d, KKLSS_FILES["keys"]), *[np.asarray(r, np.uint64) for r in rlk])
    _write_words(os.path.join(d, KKLSS_FILES["crs"]), np.asarray(crs_u, np.uint64))
    _write_words(os.path.join(d, KKLSS_FILES["output"]), np.asarray(output, np.uint64))
    order = ["0"] + [f"user{i}" for i in range(k)]
    m = _manifest(scheme, parameter, lit, k, li, level_out, beta,
                  {"input_ciphertexts_file": KKLSS_FILES["inputs"],
                   "relinearization_key_file": KKLSS_FILES["keys"], "crs_u_file": KKLSS_FILES["crs"],
                   "output_ciphertext_file": KKLSS_FILES["output"]},
                  {"ciphertext_order": order,
                   "switching_key_order": "user, relin_component[0..2], decomposition[0..beta-1], "
                                          "Q_then_P, modulus_major, coefficient_major",
                   "input_order": "side[left,right], component[0,user0..], modulus, coefficient"})
    _finish(d, m, KKLSS_FILES.values())
    return m


def _canon(a: np.ndarray, moduli) -> np.ndarray:
    a = np.array(a, dtype=np.uint64, copy=True)
    for i, q in enumerate(moduli):
        a[..., i, :] %= np.uint64(q)
    return a


def _diff(got: np.ndarray, want: np.ndarray, moduli) -> int:
    return int(np.count_nonzero(_canon(got, moduli) != _canon(want, moduli)))


def run(fix: Fixture, device: int = 0, stages: bool = True) -> dict:
    """Runs a fixture's product on the GPU through the C ABI and diffs every
    output word mod q (and the stage dumps that are present).  Returns a
    report: {"match": bool, "output_mismatches": n, "stages": {...}}."""
    from . import evaluator as ev
    lit = fix.lit
    ckks = fix.is_ckks
    P = ev.Parameters(lit, "ckks" if ckks else "bfv", device=device)
    qs = list(lit.q[: fix.level_out + 1])
    rep = {"scheme": fix.scheme, "parameter": fix.manifest.get("parameter"), "parties": fix.k,
           "stages": {}}
    scale = lit.scale if ckks else None
    if fix.scheme.startswith("MKF"):
        E = ev.MKFEvaluator(P, ev.MKFKeySet(P, list(fix.fold), fix.relin))
        left = ev.Ciphertext.from_array(P, fix.left, ckks, scale=scale)
        right = ev.Ciphertext.from_array(P, fix.right, ckks, scale=scale)
        rescale = ckks and fix.level_out < fix.level_in
        out = E.MulRelinNew(left, right, rescale=rescale, materialize=True).download()
        if out.shape[1] != fix.level_out + 1:
            raise ValueError(f"output level {out.shape[1] - 1} != fixture's {fix.level_out}")
        # ours: c0 then k gammas; the fixture: c0, gamma, then k gammas
        want = fix.expected
        mism = _diff(out[0], want[0], qs) + sum(_diff(out[1], want[j], qs) for j in range(1, fix.k + 2))
        rep["output_mismatches"] = mism
        if stages:
            rep["stages"] = _mkf_stages(fix, P)
    else:
        rs = ev.RelinearizationKeySet(P, fix.crs_u)
        for pid, words in fix.rlk.items():
            rs.AddRelinearizationKey(pid, words)
        a = ev.Ciphertext.from_array(P, fix.left, False, ids=fix.ids, scale=scale)
        b = ev.Ciphertext.from_array(P, fix.right, False, ids=fix.ids, scale=scale)
        out = ev.Evaluator(P).MulRelinNew(a, b, rs).download()
        rep["output_mismatches"] = _diff(out, fix.expected, qs)
    rep["match"] = rep["output_mismatches"] == 0 and all(
        v == 0 for v in rep["stages"].values() if isinstance(v, int))
    return rep


def _mkf_stages(fix: Fixture, P) -> dict:
    """Stage dumps of the MKF exporter (fpga_fixture_test.go:142-280) that the
    host primitives reproduce: the first switch's decomposition and ModDown,
    and both folds."""
    from . import evaluator as ev
    d, lit, ckks = fix.dir, fix.lit, fix.is_ckks
    L, N = fix.level_in, lit.n
    L1, nP = L + 1, len(lit.p)
    qs = list(lit.q[:L1])
    st = {}
    x = np.ascontiguousarray(fix.left[1])
    path = os.path.join(d, "debug_switch0_decomposition_qp.bin")
    if os.path.exists(path):
        # DecomposeNTT inverts the NTT of its input first, whatever its domain
        coeff = ev.ntt(P, x, inverse=True)
        dec = ev.decompose(P, 1, L, coeff)
        want = _read_words(path, dec.size).reshape(dec.shape)
        st["debug_switch0_decomposition_qp.bin"] = _diff(dec, want, qs + list(lit.p))
    path = os.path.join(d, "debug_switch0_moddown_q.bin")
    if os.path.exists(path):
        o0, o1 = ev.switch_one(P, L, x, fix.fold[0], in_ntt=True, ntt_output=ckks)
        want = _read_words(path, 2 * L1 * N).reshape(2, L1, N)
        st["debug_switch0_moddown_q.bin"] = _diff(np.stack([o0, o1]), want, qs)
    path = os.path.join(d, "stage_fold_q.bin")
    if os.path.exists(path):
        folds = []
        for side in (fix.left, fix.right):
            acc0 = side[0].copy() % np.array(qs, np.uint64)[:, None]
            acc1 = np.zeros_like(acc0)
            for i in range(fix.k):
                o0, o1 = ev.switch_one(P, L, side[i + 1], fix.fold[i], in_ntt=ckks, ntt_output=ckks)
                acc0, acc1 = _addmod(acc0, o0, qs), _addmod(acc1, o1, qs)
            folds += [acc0, acc1]
        want = _read_words(path, 4 * L1 * N).reshape(4, L1, N)
        st["stage_fold_q.bin"] = _diff(np.stack(folds), want, qs)
    for name in ("debug_switch0_external_qp.bin", "stage_tensor_q.bin", "stage_relinearized_q.bin",
                 "stage_rescaled_q.bin", "stage_lifted_r.bin", "stage_tensor_r.bin",
                 "stage_quantized_q.bin"):
        if os.path.exists(os.path.join(d, name)):
            st[name] = "present, not compared (covered by the final output)"
    return st


def _addmod(a: np.ndarray, b: np.ndarray, qs) -> np.ndarray:
    q = np.array(qs, np.uint64)[:, None]
    s = (a % q) + (b % q)
    return np.where(s >= q, s - q, s)


def main(argv=None):
    """python -m mkf_b200.fixtures DIR [DIR ...]: run fixture directories on
    GPU 0 and print one JSON report per directory; exit 1 on any mismatch."""
    import argparse
    import sys
    ap = argparse.ArgumentParser(prog="python -m mkf_b200.fixtures")
    ap.add_argument("dirs", nargs="+")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--no-hash-check", action="store_true")
    ap.add_argument("--no-stages", action="store_true")
    a = ap.parse_args(argv)
    ok = True
    for d in a.dirs:
        rep = run(load(d, check_hashes=not a.no_hash_check), device=a.device, stages=not a.no_stages)
        rep["dir"] = d
        print(json.dumps(rep), flush=True)
        ok = ok and rep["match"]
    sys.exit(0 if ok else 1)


if __name__ == "__main__":
    main()
