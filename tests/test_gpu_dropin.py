"""The drop-in C++ headers (second-candidate_b200/cpp) driven the way the
reference's own test drivers drive the reference classes: results match the
oracle, the `traversed` invariants hold, and the encoder writes the same
.edat_ bytes as the reference's layout."""
import os
import subprocess

import numpy as np
import pytest

import formats
import helpers
import oracle as O

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "second-candidate_b200")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    import scgpu
    scgpu.load()
    exe = str(tmp_path_factory.mktemp("drv") / "dropin_driver")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(PKG, "cpp"), "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "dropin_driver.cpp"), "-L", PKG, "-lscgpu",
                    "-Wl,-rpath," + PKG, "-o", exe], check=True)
    return exe


def parse(path):
    rows = []
    for line in open(path):
        f = line.split()
        pairs = [p.split(":") for p in f[2:]]
        rows.append((int(f[0]), int(f[1]), [int(a) for a, b in pairs], [float(b) for a, b in pairs]))
    return rows


@pytest.mark.parametrize("name,mode,tag", [("imi_d32", O.IMI, "imi"), ("sc_d32", O.SC, "sc"),
                                           ("ivf_d32", O.IVFADC, "ivf"), ("sc3_d32", O.SC3, "sc3")])
def test_search_through_dropin(driver, oracle_mod, tmp_path, name, mode, tag):
    c = helpers.load_case(os.path.join(helpers.GOLDEN, name + ".npz"))
    D, mc, kc, mp, kp = (int(c[k]) for k in ("D", "mc", "kc", "mp", "kp"))
    formats.write_ctr(tmp_path / "cq.ctr_", c["cq"], kc, mc, D)
    formats.write_ctr(tmp_path / "pq.ctr_", c["pq"], kp, mp, D)
    formats.write_edat(tmp_path / "x.edat_", c["L"], c["pid"], c["icodes"])
    formats.write_vecs(tmp_path / "q.fvecs", c["Q"])
    T, w, R = 300, (16 if mode == O.IVFADC else 1 << 12), 20
    subprocess.run([driver, "search", tag, str(tmp_path / "cq.ctr_"), str(tmp_path / "pq.ctr_"),
                    str(tmp_path / "x.edat_"), str(tmp_path / "q.fvecs"), str(D), str(R), str(w), str(T),
                    str(tmp_path / "out.txt")], check=True)
    rows = parse(tmp_path / "out.txt")
    ix = helpers.oracle_index(O, c)
    oi, od, osum = ix.search(mode, c["Q"], R, w, T, order=O.ORDER_EXACT)
    for i, (s, e, ids, d) in enumerate(rows):
        assert s == osum[i]
        m = min(R, s)
        assert ids == oi[i, :m].tolist()
        assert np.allclose(d, od[i, :m], rtol=1e-6)
        if mode == O.IMI:
            assert e == ix.search_one(mode, c["Q"][i], w, T)["empty"]


@pytest.mark.parametrize("name,mode,tag", [("imi_d32", O.IMI, "imi"), ("sc_d32", O.SC, "sc"),
                                           ("ivf_d32", O.IVFADC, "ivf")])
def test_real_dist_through_dropin(driver, oracle_mod, tmp_path, name, mode, tag):
    """real_dist = true after load_data: every candidate of the visited cells
    scored by its exact distance (query.h:307-312, multi_query.h:255-259,
    sc_query.h:232-236), the R best returned -- the oracle's real_dist
    branch in the exact order, bit for bit."""
    c = helpers.load_case(os.path.join(helpers.GOLDEN, name + ".npz"))
    D, mc, kc, mp, kp = (int(c[k]) for k in ("D", "mc", "kc", "mp", "kp"))
    formats.write_ctr(tmp_path / "cq.ctr_", c["cq"], kc, mc, D)
    formats.write_ctr(tmp_path / "pq.ctr_", c["pq"], kp, mp, D)
    formats.write_edat(tmp_path / "x.edat_", c["L"], c["pid"], c["icodes"])
    formats.write_vecs(tmp_path / "q.fvecs", c["Q"])
    formats.write_vecs(tmp_path / "x.fvecs", c["X"].astype(np.float32))
    T, w, R = 300, (16 if mode == O.IVFADC else 1 << 16), 20
    subprocess.run([driver, "search", tag, str(tmp_path / "cq.ctr_"), str(tmp_path / "pq.ctr_"),
                    str(tmp_path / "x.edat_"), str(tmp_path / "q.fvecs"), str(D), str(R), str(w), str(T),
                    str(tmp_path / "out.txt"), str(tmp_path / "x.fvecs")], check=True)
    rows = parse(tmp_path / "out.txt")
    ix = helpers.oracle_index(O, c)
    oi, od, osum = ix.search(mode, c["Q"], R, w, T, order=O.ORDER_EXACT, real_dist=True)
    for i, (s, e, ids, d) in enumerate(rows):
        assert s == osum[i]
        m = min(R, s)
        assert helpers.same_topk(np.array(ids), np.array(d, np.float32), oi[i], od[i], m)


@pytest.mark.parametrize("name,nc", [("imi_d32", 0), ("sc_d32", 2)])
def test_encoder_through_dropin(driver, oracle_mod, tmp_path, name, nc):
    c = helpers.load_case(os.path.join(helpers.GOLDEN, name + ".npz"))
    D, mc, kc, mp, kp = (int(c[k]) for k in ("D", "mc", "kc", "mp", "kp"))
    formats.write_ctr(tmp_path / "cq.ctr_", c["cq"], kc, mc, D)
    formats.write_ctr(tmp_path / "pq.ctr_", c["pq"], kp, mp, D)
    formats.write_vecs(tmp_path / "x.fvecs", c["X"].astype(np.float32))
    subprocess.run([driver, "encode", str(nc), str(tmp_path / "cq.ctr_"), str(tmp_path / "pq.ctr_"),
                    str(tmp_path / "x.fvecs"), str(tmp_path), "d"], check=True)
    got = open(tmp_path / ("d_mr2_ivf.edat_" if nc else "d_ivf.edat_"), "rb").read()
    formats.write_edat(tmp_path / "ref.edat_", c["L"], c["pid"], c["icodes"])
    assert got == open(tmp_path / "ref.edat_", "rb").read()


def test_quantizer_through_dropin(driver, oracle_mod, tmp_path):
    """PQQuantizer (drop-in): trains the strips on the GPU, writes a .ctr_
    with the reference's header, deterministic, and prints the reference's
    distortion formula for the final assignment; calc_residual_vector of
    PQQuantizer / SCQuantizer subtracts the nearest / second-nearest
    centroid per part."""
    import workloads as W
    D, m, nsc = 32, 4, 64
    mix = W.Mixture(D, 8, 20.0, "u8", seed=121)
    X = mix.sample(5000, seed=122)
    formats.write_vecs(tmp_path / "x.fvecs", X)
    outs = []
    for run in range(2):
        r = subprocess.run([driver, "quantize", str(tmp_path / "x.fvecs"), str(D), str(m), str(nsc),
                            str(tmp_path / ("cb%d" % run))], check=True, capture_output=True, text=True)
        outs.append((float(r.stdout.split()[-1]), open(tmp_path / ("cb%d.ctr_" % run), "rb").read()))
    assert outs[0][1] == outs[1][1]  # deterministic
    raw = np.frombuffer(outs[0][1], np.float32)
    assert raw[:3].tolist() == [nsc, m, D] and raw.size == 3 + nsc * D
    C = raw[3:].reshape(m, nsc, D // m).astype(np.float64)
    e = 0.0
    for i in range(m):
        part = X[:, i * (D // m):(i + 1) * (D // m)].astype(np.float64)
        d = ((part[:, None, :] - C[i][None]) ** 2).sum(2).min(1)
        e += d.sum()
    assert abs(outs[0][0] - np.sqrt(e)) <= 1e-3 * np.sqrt(e)
    # residuals against a 2-part coarse codebook
    cq = np.asarray(W.train_codebooks(X[:2000], 2, 16, 4, 8, 2, seed=123)[0], np.float32)
    formats.write_ctr(tmp_path / "cq.ctr_", cq, 16, 2, D)
    for kind in ("pq", "sc"):
        subprocess.run([driver, "residual", kind, str(tmp_path / "x.fvecs"), str(D), "2", str(tmp_path / "cq.ctr_"),
                        str(tmp_path / "r.fvecs")], check=True)
        Rr = formats.read_vecs(tmp_path / "r.fvecs", np.float32)
        for i in range(2):
            part = X[:, i * 16:(i + 1) * 16]
            diff = (part[:, None, :] - cq[i][None]).astype(np.float64)  # float differences, double squares
            d = (diff ** 2).sum(2).astype(np.float32)
            order = np.argsort(d, axis=1, kind="stable")
            pick = order[:, 0] if kind == "pq" else order[:, 1]
            assert np.array_equal(Rr[:, i * 16:(i + 1) * 16], part - cq[i][pick]), kind
