"""OBJ loading (src/BaseModel.cpp:3-25): the oracle's reading of the
reference, and the product loader against the oracle."""
import numpy as np
import pytest


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_bytes(text.encode() if isinstance(text, str) else text)
    return str(p)


CASES = {
    "plain": "v 0 0 0\nv 1 0 0\nv 0 1 0\nv 0 0 1\nf 1 2 3\nf 1 3 4\n",
    "double_slash": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1//7 2//8 3//9\n",
    "tex": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1/5 2/6 3/7\n",
    # a/t/n faces match none of the reference's patterns and are dropped
    "tex_normal": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1/1/1 2/2/2 3/3/3\nf 1 2 3\n",
    # quads keep their first triangle
    "quad": "v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0\nf 1 2 4 3\n",
    # vn / vt / comments / tabs after v are ignored
    "other_lines": "# c\nvn 1 0 0\nvt 0 0\nv\t5 5 5\nv 0 0 0\nv 1 0 0\nv 0 1 0\n\nf 1 2 3\n",
    # unterminated last line is dropped
    "unterminated": "v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\nv 9 9 9",
    "crlf": "v 0 0 0\r\nv 1 0 0\r\nv 0 1 0\r\nf 1 2 3\r\n",
    "short_v": "v 1 2\nv 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3\n",
    "exp_floats": "v 1e-3 -2.5E+2 +7\nv 0.1 0.2 0.30000001\nv 3 nan 4\nf 1 2 3\n",
    "spaces": "v   1   2   3\nv 0 0 0\nv 1 1 1\nf  1  2  3\n",
    "line_254": "v 1 2 3" + " " * 247 + "\nv 0 0 0\nv 1 1 1\nf 1 2 3\n",
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_loader_cases(tmp_path, oracle_mod, name):
    path = _write(tmp_path, name + ".obj", CASES[name])
    pts, tri = oracle_mod.load_obj(path)
    if name == "tex_normal":
        assert tri.tolist() == [[0, 1, 2]]
    if name == "quad":
        assert tri.tolist() == [[0, 1, 3]]
    if name == "other_lines":
        assert pts.shape == (3, 3) and tri.shape == (1, 3)
    if name == "unterminated":
        assert pts.shape == (3, 3) and tri.shape == (1, 3)
    if name == "short_v":
        assert pts.shape == (3, 3)
    if name == "exp_floats":
        assert pts[0].tolist() == [np.float32(1e-3), -250.0, 7.0]
        assert np.isnan(pts[2, 1])


@pytest.mark.parametrize("name", sorted(CASES))
def test_product_loader_matches_oracle(tmp_path, oracle_mod, svo_mod, name):
    path = _write(tmp_path, name + ".obj", CASES[name])
    p0, t0 = oracle_mod.load_obj(path)
    p1, t1 = svo_mod.load_obj(path)
    assert p0.tobytes() == p1.tobytes()
    assert np.array_equal(t0, t1)


@pytest.mark.parametrize("text,code", [
    ("v 0 0 0\n" + "v " + "1 " * 130 + "\n", 7),          # 255+ characters: reference never returns
    ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 9\n", 7),           # index past the vertex list
    ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 0 1 2\n", 7),           # index 0 -> -1
])
def test_loader_errors(tmp_path, oracle_mod, svo_mod, text, code):
    path = _write(tmp_path, "bad.obj", text)
    with pytest.raises(oracle_mod.OracleError) as e0:
        oracle_mod.load_obj(path)
    with pytest.raises(svo_mod.SvoError) as e1:
        svo_mod.load_obj(path)
    assert e0.value.code == code and e1.value.code == code


def test_missing_file(oracle_mod, svo_mod, tmp_path):
    with pytest.raises(svo_mod.SvoError) as e:
        svo_mod.load_obj(str(tmp_path / "nope.obj"))
    assert e.value.code == svo_mod.ERR_IO


def test_bunny(bunny_path, oracle_mod, svo_mod):
    p0, t0 = oracle_mod.load_obj(bunny_path)
    p1, t1 = svo_mod.load_obj(bunny_path)
    assert p0.shape == (14290, 3) and t0.shape == (28576, 3)
    assert p0.tobytes() == p1.tobytes() and np.array_equal(t0, t1)


def _big_obj(seed, n_v, n_f):
    """A multi-megabyte OBJ mixing every line form the loader meets (so the
    product loader cuts it into chunks parsed in parallel)."""
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n_v, 3)).astype(np.float32)
    f = rng.integers(1, n_v + 1, size=(n_f, 3))
    out = ["# generated\n"]
    vi = fi = 0
    while vi < n_v or fi < n_f:
        r = rng.integers(0, 12)
        if vi < n_v and (r < 5 or fi >= n_f):
            x, y, z = (float(c) for c in v[vi])
            sep = " " if r else "   "
            out.append(f"v{sep}{x!r}{sep}{y:.9g} {z:.3e}\n" if r % 2 else f"v {x} {y} {z}\r\n")
            vi += 1
        elif fi < n_f and vi >= max(f[fi]):  # faces only after their vertices (any order is valid)
            a, b, c = f[fi]
            form = rng.integers(0, 4)
            out.append([f"f {a} {b} {c}\n", f"f {a}//{a} {b}//{b} {c}//{c}\n", f"f {a}/1 {b}/2 {c}/3\n",
                        f"f {a}/1/1 {b}/2/2 {c}/3/3\n"][form])
            fi += 1
        elif r < 8:
            out.append(["vn 0 0 1\n", "vt 0.5 0.5\n", "\n", "# " + "x" * 200 + "\n"][r - 5 if r < 8 else 0])
        elif vi < n_v:
            x, y, z = (float(c) for c in v[vi])
            out.append(f"v {x} {y} {z}\n")
            vi += 1
        else:
            a, b, c = f[fi]
            out.append(f"f {a} {b} {c}\n")
            fi += 1
    return "".join(out)


def test_big_file_matches_oracle(tmp_path, oracle_mod, svo_mod):
    text = _big_obj(11, 60000, 120000)
    assert len(text) > 4 << 20
    for name, t in (("big.obj", text), ("big_unterminated.obj", text + "v 1 2 3")):
        path = _write(tmp_path, name, t)
        p0, t0 = oracle_mod.load_obj(path)
        p1, t1 = svo_mod.load_obj(path)
        assert p0.shape[0] == 60000 and t0.shape[0] > 80000
        assert p0.tobytes() == p1.tobytes() and np.array_equal(t0, t1)


def test_big_file_errors(tmp_path, oracle_mod, svo_mod):
    text = _big_obj(12, 40000, 80000)
    mid = text.index("\n", len(text) * 2 // 3) + 1
    for bad, code in (("v " + "1 " * 130 + "\n", 7), ("f 1 2 999999\n", 7)):
        path = _write(tmp_path, "bad_big.obj", text[:mid] + bad + text[mid:])
        with pytest.raises(oracle_mod.OracleError) as e0:
            oracle_mod.load_obj(path)
        with pytest.raises(svo_mod.SvoError) as e1:
            svo_mod.load_obj(path)
        assert e0.value.code == code and e1.value.code == code


@pytest.mark.parametrize("mb", [0.25, 0.5, 1.0, 2.0, 3.3])
def test_chunk_cuts(tmp_path, oracle_mod, svo_mod, mb):
    """Files around the loader's 256 KB chunk size, made of maximal (254
    character) vertex lines, CRLF lines and faces in every form, so that the
    cut points fall inside lines of each kind."""
    target = int(mb * (1 << 20))
    out, nv, size = [], 0, 0
    k = 0
    while size < target:
        r = k % 5
        if r == 0:
            line = "v 1 2 3" + " " * 246 + "\n"       # 254 characters + newline
            nv += 1
        elif r == 1:
            line = f"v {k * 0.5} {-k} 1e-3\r\n"
            nv += 1
        elif r == 2 and nv >= 3:
            line = f"f {nv} {nv - 1} {nv - 2}\n"
        elif r == 3 and nv >= 3:
            line = f"f {nv}//1 {nv - 1}//2 {nv - 2}//3\n"
        else:
            line = f"f {nv}/4 {max(1, nv - 2)}/5 {max(1, nv - 1)}/6\n" if nv >= 3 else "# start\n"
        out.append(line)
        size += len(line)
        k += 1
    path = _write(tmp_path, "cuts.obj", "".join(out))
    p0, t0 = oracle_mod.load_obj(path)
    p1, t1 = svo_mod.load_obj(path)
    assert p0.tobytes() == p1.tobytes() and np.array_equal(t0, t1)
    assert t0.shape[0] > 0


def test_empty_and_blank_files(tmp_path, oracle_mod, svo_mod):
    for name, text in (("empty.obj", ""), ("blank.obj", "\n" * 300000), ("comments.obj", "# x\n" * 100000)):
        path = _write(tmp_path, name, text)
        p0, t0 = oracle_mod.load_obj(path)
        p1, t1 = svo_mod.load_obj(path)
        assert p0.shape == p1.shape == (0, 3) and t0.shape == t1.shape == (0, 3)
