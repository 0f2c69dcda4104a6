"""Writes proof_digests.json: SHA-256 digests of full-size oracle proofs.

For each reference parameter set named on the command line (default: A0, A1,
A2, F0, F1, F2; the presets of src/protocol.rs:28-123) the CPU oracle proves
one statement at a fixed (crs_seed, seed) with the witness sampled from the
seed, checks the proof with its own verifier (the reference verifier's checks),
and records the proof length and the SHA-256 of its bytes.  The GPU tests
prove the same statements and compare digests, so a full-size proof is
checked byte for byte without the oracle running on the GPU box (an A0 proof
takes about a minute on 16 host cores, F2 about a quarter of an hour).

Usage: python tests/golden/make_proof_digests.py [--threads N] [NAME ...]
Existing entries for other presets are kept.
"""
import hashlib
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

OUT = os.path.join(HERE, "proof_digests.json")
CRS_SEED = 1
SEED = 2
DEFAULT = ["A0", "A1", "A2", "F0", "F1", "F2"]


def digest(proof_bytes):
    return hashlib.sha256(bytes(proof_bytes)).hexdigest()


def main(argv):
    import oracle as O
    from salsaa_b200 import params as P

    threads = 0
    names = []
    it = iter(argv)
    for a in it:
        if a == "--threads":
            threads = int(next(it))
        else:
            names.append(a)
    names = names or DEFAULT
    table = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            table = json.load(f)
    for name in names:
        p = P.preset(name)
        t0 = time.time()
        rc, proof, _ = O.prove(p, CRS_SEED, SEED, nthreads=threads)
        if rc != 0:
            raise SystemExit("oracle prove failed for %s (%d)" % (name, rc))
        verdict = O.verify(p, CRS_SEED, SEED, proof)
        if verdict != 0:
            raise SystemExit("oracle verifier rejected %s (%d)" % (name, verdict))
        table[name] = {"crs_seed": CRS_SEED, "seed": SEED, "bytes": int(proof.size), "sha256": digest(proof),
                       "params": p.as_dict()}
        print("%s: %d bytes, %s, %.1f s" % (name, proof.size, table[name]["sha256"][:16], time.time() - t0),
              flush=True)
        with open(OUT, "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
            f.write("\n")


if __name__ == "__main__":
    main(sys.argv[1:])
