"""Generate the golden fixtures in tests/golden/ from the reference CUDA-ORB build.

Runs the reference's own orbd.cu/orb.cpp (compiled for sm_100a into
oracle/_ref/libref_orb.so by `make -C oracle ref`) on seeded synthetic inputs
and stores its outputs as compressed .npz files.  Needs a GPU.

    python tests/golden/make_golden.py [out_dir]

Fixtures:
  pair_320x240_s1.npz   images A/B, per image: race-free staged outputs (raw and
                        blurred pyramid, sparse score map, points, descriptors,
                        __sinf/__cosf of each angle), stock Orbor outputs, and
                        the A->B matches of both.
  pair_640x480_s2.npz   same without the pyramids.
  variants_320x240.npz  FAST score, WTA_K 3 and 4, patch size 25.
  cap_320x240.npz       keypoint cap far below the survivor count.
  match_kat.npz         hand-made descriptor sets for the matcher semantics.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "cuda-orb_b200"))
sys.path.insert(0, ROOT)

import synth  # noqa: E402
from oracle import refharness as ref  # noqa: E402


def sparse_map(st):
    nz = np.nonzero(st["vmap"])[0].astype(np.int64)
    return nz, st["vmap"][nz].copy(), st["layer"][nz].copy()


def image_record(prefix, img, w, h, max_pts, keep_pyramids, out):
    st = ref.stages(img, w, h, max_pts, race_free=True)
    out[prefix + "num_pts"] = np.int64(st["num_pts"])
    out[prefix + "raw_counter"] = np.int64(st["raw_counter"])
    out[prefix + "points"] = st["points"]
    out[prefix + "desc"] = st["desc"]
    out[prefix + "sin"] = st["sin"]
    out[prefix + "cos"] = st["cos"]
    idx, sc, ly = sparse_map(st)
    out[prefix + "map_idx"] = idx
    out[prefix + "map_score"] = sc
    out[prefix + "map_layer"] = ly
    if keep_pyramids:
        out[prefix + "pyr_raw"] = st["pyr_raw"]
        out[prefix + "pyr_blur"] = st["pyr_blur"]
    stock = ref.stages(img, w, h, max_pts, race_free=False)
    out[prefix + "stock_points"] = stock["points"]
    out[prefix + "stock_desc"] = stock["desc"]
    return st, stock


def pair_fixture(path, w, h, seed, max_pts, keep_pyramids):
    a, b, H = synth.make_pair(w, h, seed)
    ref.init(noctaves=8, edge=31, wta_k=2, score_type=0, patch=31, fast_thr=20, retain_topn=-1, max_pts=max_pts)
    out = {"imgA": a, "imgB": b, "H": H, "w": np.int64(w), "h": np.int64(h), "max_pts": np.int64(max_pts)}
    lay = ref.layout_for(w, h, 8)
    out["oszp"] = np.concatenate([lay["osizes"], lay["widths"], lay["heights"], lay["pitchs"], lay["offsets"]])
    sa, ka = image_record("A_", a, w, h, max_pts, keep_pyramids, out)
    sb, kb = image_record("B_", b, w, h, max_pts, keep_pyramids, out)
    m, d = ref.hmatch(sa["desc"], sb["desc"])
    out["match_rf"], out["dist_rf"] = m, d
    m, d = ref.hmatch(ka["desc"], kb["desc"])
    out["match_stock"], out["dist_stock"] = m, d
    # the stock Orbor path end to end (detectAndCompute x2 + match)
    ra = ref.detect(0, a, w, h, max_pts)
    rb = ref.detect(1, b, w, h, max_pts)
    m, d = ref.match_slots(ra["num_pts"])
    out["orbor_A_points"], out["orbor_A_desc"] = ra["points"], ra["desc"]
    out["orbor_B_points"], out["orbor_B_desc"] = rb["points"], rb["desc"]
    out["orbor_match"], out["orbor_dist"] = m, d
    np.savez_compressed(path, **out)
    print(f"{os.path.basename(path)}: A {sa['num_pts']} pts (counter {sa['raw_counter']}), "
          f"B {sb['num_pts']} pts, race-affected desc rows A: "
          f"{int(np.any(sa['desc'] != ka['desc'], axis=1).sum()) if sa['num_pts'] == ka['num_pts'] else 'n/a'}")


def variants_fixture(path):
    w, h = 320, 240
    img = synth.make_image(w, h, 3)
    out = {"img": img, "w": np.int64(w), "h": np.int64(h)}
    cases = {
        "fast": dict(score_type=1, wta_k=2, patch=31),
        "wta3": dict(score_type=0, wta_k=3, patch=31),
        "wta4": dict(score_type=0, wta_k=4, patch=31),
        "patch25": dict(score_type=0, wta_k=2, patch=25),
    }
    for name, c in cases.items():
        ref.init(noctaves=8, edge=31, fast_thr=20, retain_topn=-1, max_pts=4000, **c)
        st = ref.stages(img, w, h, 4000, race_free=True)
        out[name + "_points"] = st["points"]
        out[name + "_desc"] = st["desc"]
        out[name + "_sin"] = st["sin"]
        out[name + "_cos"] = st["cos"]
        idx, sc, ly = sparse_map(st)
        out[name + "_map_idx"], out[name + "_map_score"], out[name + "_map_layer"] = idx, sc, ly
        print(f"variant {name}: {st['num_pts']} pts")
    np.savez_compressed(path, **out)


def cap_fixture(path):
    w, h = 320, 240
    img = synth.make_image(w, h, 4)
    out = {"img": img, "w": np.int64(w), "h": np.int64(h)}
    ref.init(noctaves=8, edge=31, wta_k=2, score_type=0, patch=31, fast_thr=20, retain_topn=-1, max_pts=40)
    st = ref.stages(img, w, h, 40, race_free=True)
    out["cap"] = np.int64(40)
    out["cap_num_pts"] = np.int64(st["num_pts"])
    out["cap_raw_counter"] = np.int64(st["raw_counter"])
    out["cap_points"] = st["points"]
    ref.init(noctaves=8, edge=31, wta_k=2, score_type=0, patch=31, fast_thr=20, retain_topn=-1, max_pts=10000)
    full = ref.stages(img, w, h, 10000, race_free=True)
    out["full_points"] = full["points"]
    np.savez_compressed(path, **out)
    print(f"cap: {st['num_pts']} kept of counter {st['raw_counter']}, full {full['num_pts']}")


def flip_bits(d, nbits, rng):
    d = d.copy()
    pos = rng.choice(256, size=nbits, replace=False)
    for p in pos:
        d[p // 8] ^= np.uint8(1 << (p % 8))
    return d


def match_kat_fixture(path):
    rng = np.random.Generator(np.random.PCG64(77))
    out = {}
    cases = []
    q = rng.integers(0, 256, size=(37, 32), dtype=np.uint8)
    cases.append(("n2_0", q, np.zeros((0, 32), dtype=np.uint8)))
    # n2 = 1 at exact distances 0, 1, 63, 64, 65, 256
    base = rng.integers(0, 256, size=(1, 32), dtype=np.uint8)
    qs = np.stack([flip_bits(base[0], k, rng) for k in (0, 1, 63, 64, 65, 256)])
    cases.append(("n2_1", qs, base))
    # ties: the nearest train row appears twice; and distinct rows at equal distance
    db = rng.integers(0, 256, size=(50, 32), dtype=np.uint8)
    db[17] = db[3]
    qt = np.stack([flip_bits(db[3], k, rng) for k in (0, 5, 40, 63)] +
                  [flip_bits(db[8], 10, rng)])
    cases.append(("ties", qt, db))
    db2 = rng.integers(0, 256, size=(40, 32), dtype=np.uint8)
    q2 = db2[:8].copy()
    db2[20:28] = np.stack([flip_bits(db2[i], 2, rng) for i in range(8)])
    qa = np.stack([flip_bits(db2[i], 1, rng) for i in range(8)])
    cases.append(("equal_dist", np.concatenate([q2, qa]), db2))
    # random sets with planted near matches, several sizes incl. n not a multiple of 32
    for n1, n2 in ((1, 1), (33, 31), (500, 700), (1000, 1000)):
        dbr = rng.integers(0, 256, size=(n2, 32), dtype=np.uint8)
        qr = rng.integers(0, 256, size=(n1, 32), dtype=np.uint8)
        k = n1 // 2
        src = rng.integers(0, n2, size=k)
        for i in range(k):
            qr[i] = flip_bits(dbr[src[i]], int(rng.integers(0, 70)), rng)
        cases.append((f"rand_{n1}x{n2}", qr, dbr))
    for name, a, b in cases:
        m, d = ref.hmatch(a, b)
        out[name + "_q"], out[name + "_db"], out[name + "_match"], out[name + "_dist"] = a, b, m, d
        print(f"kat {name}: {len(a)}x{len(b)}, matched {(m >= 0).sum()}")
    out["names"] = np.array([c[0] for c in cases])
    np.savez_compressed(path, **out)


def main():
    out_dir = sys.argv[1] if len(sys.argv) > 1 else os.path.dirname(os.path.abspath(__file__))
    os.makedirs(out_dir, exist_ok=True)
    pair_fixture(os.path.join(out_dir, "pair_320x240_s1.npz"), 320, 240, 1, 10000, True)
    pair_fixture(os.path.join(out_dir, "pair_640x480_s2.npz"), 640, 480, 2, 10000, False)
    variants_fixture(os.path.join(out_dir, "variants_320x240.npz"))
    cap_fixture(os.path.join(out_dir, "cap_320x240.npz"))
    match_kat_fixture(os.path.join(out_dir, "match_kat.npz"))


if __name__ == "__main__":
    main()
