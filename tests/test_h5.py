"""HDF5 / XDMF output (the reference's write_output.f90 layouts) and the
classic-format reader, on the CPU.

No HDF5 library exists here, so the files are checked by an independent
minimal parser written in this test from the HDF5 File Format
Specification.  That parser is first validated on a file the real HDF5
library wrote (a MATLAB 7.3 test file shipped with scipy, compared with
scipy's MATLAB 5 copy of the same variable), then applied to our files."""
import os
import struct

import numpy as np
import pytest

import scarl_b200 as S

SIG = b"\x89HDF\r\n\x1a\n"
SCIPY_DATA = None
try:
    import scipy.io
    SCIPY_DATA = os.path.join(os.path.dirname(scipy.io.__file__), "matlab", "tests", "data")
except Exception:  # pragma: no cover
    pass


# ---------------------------------------------------------------------------
# independent parser (classic format: superblock 0, v1 headers, symbol tables)
# ---------------------------------------------------------------------------
class H5:
    def __init__(self, path):
        self.b = open(path, "rb").read()
        self.sb = next(o for o in (0, 512, 1024, 2048) if self.b[o:o + 8] == SIG)
        b, o = self.b, self.sb
        self.version = b[o + 8]
        assert self.version == 0
        self.sizes = (b[o + 13], b[o + 14])
        self.leafK, self.intK = struct.unpack_from("<HH", b, o + 16)
        self.base, self.freespace, self.eof, self.driver = struct.unpack_from("<QQQQ", b, o + 24)
        _, self.root_oh, cache, _, tree, heap = struct.unpack_from("<QQIIQQ", b, o + 56)
        self.root_msgs = self.messages(self.root_oh)
        st = [m for t, m in self.root_msgs if t == 0x11][0]
        self.tree, self.heap = struct.unpack_from("<QQ", st)
        assert (cache, tree, heap) == (1, self.tree, self.heap)
        h = self.base + self.heap
        assert b[h:h + 4] == b"HEAP"
        self.heap_size, self.free_head, hd = struct.unpack_from("<QQQ", b, h + 8)
        self.heap_data = b[self.base + hd:self.base + hd + self.heap_size]
        self.entries = self.walk(self.tree)
        self.root_attrs = self.attrs(self.root_msgs)

    def messages(self, rel):
        b, a = self.b, self.base + rel
        assert b[a] == 1
        n, _, size = struct.unpack_from("<HII", b, a + 2)
        out, off = [], a + 16
        end = off + size
        while off < end and len(out) < n:
            t, sz, _ = struct.unpack_from("<HHB", b, off)
            assert sz % 8 == 0
            out.append((t, b[off + 8:off + 8 + sz]))
            off += 8 + sz
        assert len(out) == n
        return out

    def name(self, off):
        return self.heap_data[off:self.heap_data.index(b"\0", off)].decode()

    def walk(self, rel):
        b, a = self.b, self.base + rel
        assert b[a:a + 4] == b"TREE" and b[a + 4] == 0
        level, used = b[a + 5], struct.unpack_from("<H", b, a + 6)[0]
        keys = [struct.unpack_from("<Q", b, a + 24 + 16 * i)[0] for i in range(used + 1)]
        kids = [struct.unpack_from("<Q", b, a + 32 + 16 * i)[0] for i in range(used)]
        out = []
        for i, c in enumerate(kids):
            if level:
                out += self.walk(c)
                continue
            s = self.base + c
            assert b[s:s + 4] == b"SNOD" and b[s + 4] == 1
            n = struct.unpack_from("<H", b, s + 6)[0]
            names = []
            for e in range(n):
                noff, oh = struct.unpack_from("<QQ", b, s + 8 + 40 * e)
                names.append(self.name(noff))
                out.append((self.name(noff), oh))
            # group B-tree keys bound each child's names
            assert names == sorted(names)
            assert self.name(keys[i + 1]) == names[-1]
        return out

    @staticmethod
    def dtype(m):
        cls, size = m[0] & 15, struct.unpack_from("<I", m, 4)[0]
        if cls == 1:
            return np.dtype("<f%d" % size), size
        if cls == 0:
            return np.dtype("<i%d" % size), size
        assert cls == 3
        return "S%d" % size, size

    @staticmethod
    def space(m):
        assert m[0] == 1
        rank = m[1]
        return tuple(struct.unpack_from("<%dQ" % rank, m, 8)) if rank else ()

    def attrs(self, msgs):
        out = {}
        for t, m in msgs:
            if t != 0xC:
                continue
            assert m[0] == 1
            nl, dl, sl = struct.unpack_from("<HHH", m, 2)
            up = lambda x: (x + 7) // 8 * 8
            off = 8
            name = m[off:off + nl - 1].decode()
            off += up(nl)
            dt, sz = self.dtype(m[off:off + dl])
            off += up(dl)
            dims = self.space(m[off:off + sl])
            off += up(sl)
            cnt = int(np.prod(dims)) if dims else 1
            raw = m[off:off + cnt * sz]
            out[name] = raw if isinstance(dt, str) else np.frombuffer(raw, dt)
        return out

    def dataset(self, name):
        rel = dict(self.entries)[name]
        msgs = self.messages(rel)
        dt = dims = addr = size = None
        for t, m in msgs:
            if t == 0x3:
                dt, _ = self.dtype(m)
            elif t == 0x1:
                dims = self.space(m)
            elif t == 0x8:
                if m[0] == 3:
                    assert m[1] == 1
                    addr, size = struct.unpack_from("<QQ", m, 2)
                else:  # layout v1/v2 (older writers)
                    nd = m[1]
                    addr = struct.unpack_from("<Q", m, 8)[0]
                    size = int(np.prod(struct.unpack_from("<%dI" % nd, m, 16)))
        raw = self.b[self.base + addr:self.base + addr + size]
        if isinstance(dt, str):
            return raw, dims, self.attrs(msgs)
        return np.frombuffer(raw, dt).reshape(dims), dims, self.attrs(msgs)


REAL = None if SCIPY_DATA is None else os.path.join(SCIPY_DATA, "testhdf5_7.4_GLNX86.mat")


@pytest.mark.skipif(REAL is None or not os.path.exists(REAL), reason="no library-written HDF5 file")
def test_parsers_read_a_file_written_by_the_hdf5_library():
    ref = scipy.io.loadmat(os.path.join(SCIPY_DATA, "testdouble_7.4_GLNX86.mat"))["testdouble"]
    f = H5(REAL)
    assert f.sb == 512 and f.base == 512 and (f.leafK, f.intK) == (4, 16)
    assert [e[0] for e in f.entries] == ["testdouble"]
    data, dims, attrs = f.dataset("testdouble")
    assert attrs["MATLAB_class"] == b"double"
    # HDF5 dims are the MATLAB (column-major) shape reversed
    np.testing.assert_array_equal(data.reshape(ref.shape[::-1]).T, ref)
    assert S.h5_list(REAL) == ["testdouble"]
    got = S.h5_read_dataset(REAL, "testdouble")
    np.testing.assert_array_equal(got.reshape(ref.shape), ref)


def _deck(topo=(2, 2, 1)):
    s = S.make_sample((0, 0, 0), (19, 14, 9), (4, 3, 2), (1, 1, 1), (5, 4, 3), corrMod=1,
                      margiFirst=2, avg=1.0, std_dev=0.2, seedBase=7)
    nb = int(np.prod(topo))
    return s, S.sample_layout(s, 1, nb, topo)


def _field(lay, dtype=np.float64, seed=0):
    L = tuple(int(v) for v in lay["L"])
    return np.asfortranarray(np.random.default_rng(seed).standard_normal(L).astype(dtype))


def test_one_file_one_dataset_layout(tmp_path):
    s, lay = _deck()
    f = _field(lay)
    S.write_sample_h5(None, tmp_path, "RF", f, s, lay, times=[0.5, 1.25, 2.0],
                      time_labels=["Generation", "Apply_unit", "Total_Wall_time"])
    path = tmp_path / "RF.h5"
    h = H5(path)
    assert h.sizes == (8, 8) and h.base == 0 and h.eof == os.path.getsize(path)
    assert h.free_head < h.heap_size
    assert struct.unpack_from("<Q", h.heap_data, h.free_head)[0] == 1  # end of the free list
    assert [e[0] for e in h.entries] == ["samples", "time_labels", "times"]
    data, dims, attrs = h.dataset("samples")
    L = [int(v) for v in lay["L"]]
    assert dims == (L[2], L[1], L[0]) and data.dtype == np.float64
    np.testing.assert_array_equal(data.ravel(), f.ravel(order="F"))
    np.testing.assert_array_equal(attrs["pos_0"], [1, 1, 1])
    np.testing.assert_array_equal(attrs["pos_N"], L)
    np.testing.assert_array_equal(attrs["xMin"], [0, 0, 0])
    xs = np.asarray(lay["xStep"])
    np.testing.assert_allclose(attrs["xMax"], (np.array(L) - 1) * xs)
    ra = h.root_attrs
    assert int(ra["nb_procs"][0]) == 4 and int(ra["nDim"][0]) == 3 and int(ra["Nmc"][0]) == 1
    assert int(ra["method"][0]) == 1 and int(ra["seedStart"][0]) == 7
    assert int(ra["corrMod"][0]) == 1 and int(ra["margiFirst"][0]) == 2
    np.testing.assert_array_equal(ra["nFields"], lay["topo"])
    for k in ("Np", "Np_ovlp", "L"):
        np.testing.assert_array_equal(ra[k], lay[k])
    np.testing.assert_array_equal(ra["xStep"], xs)
    np.testing.assert_array_equal(ra["corrL"], [4, 3, 2])
    np.testing.assert_allclose(ra["overlap"], (np.asarray(lay["Np_ovlp"]) - 1) * xs)
    t, tdims, _ = h.dataset("times")
    assert tdims == (1, 3)
    np.testing.assert_array_equal(t.ravel(), [0.5, 1.25, 2.0])
    lab, ldims, _ = h.dataset("time_labels")
    assert ldims == (3,) and lab == b"Generation          Apply_unit          Total_Wall_time     "
    # the library's own reader agrees
    np.testing.assert_array_equal(S.h5_read_dataset(path, "samples"), f)
    np.testing.assert_array_equal(S.h5_read_attr(path, "L"), L)
    np.testing.assert_array_equal(S.h5_read_attr(path, "pos_N", "samples"), L)
    # XDMF companion
    x = (tmp_path / "RF.xmf").read_text().splitlines()
    dt = "%d %d %d" % (L[2], L[1], L[0])
    assert x[0] == '<?xml version="1.0" ?>' and x[1] == '<Xdmf Version="2.0">'
    assert x[3] == ('   <DataItem Name="RF_1" Format="HDF" DataType="Float" Precision="8" '
                    'Dimensions="%s">' % dt)
    assert x[4] == "        ./RF.h5:/samples"
    assert '<Topology TopologyType="3DCoRectMesh" Dimensions="%s"/>' % dt in x[8]
    step = [float(v) for v in x[16:19]]
    np.testing.assert_allclose(step, xs[::-1])
    assert x[16] == " %25.10f" % xs[2]


def test_one_file_per_tile_datasets_many_symbol_nodes(tmp_path):
    s, lay = _deck((3, 2, 2))  # 12 tiles: two symbol table nodes, names out of numeric order
    f = _field(lay, np.float32, 3)
    S.write_sample_h5(None, tmp_path, "RF", f, s, lay, one_file=True, one_hdf_ds=False)
    h = H5(tmp_path / "RF.h5")
    names = [e[0] for e in h.entries]
    assert names == sorted("sample_1_p%d" % r for r in range(12))
    Np = [int(v) for v in lay["Np"]]
    for r in range(12):
        g = S.tile_geometry(lay, (0, 0, 0), r)
        o = np.asarray(g["pos_0"]) - 1
        data, dims, attrs = h.dataset("sample_1_p%d" % r)
        assert dims == (Np[2], Np[1], Np[0]) and data.dtype == np.float32
        blk = f[o[0]:o[0] + Np[0], o[1]:o[1] + Np[1], o[2]:o[2] + Np[2]]
        np.testing.assert_array_equal(data.ravel(), blk.ravel(order="F"))
        np.testing.assert_array_equal(attrs["pos_0"], g["pos_0"])
        np.testing.assert_array_equal(attrs["xMin"], g["coord_0"])
    x = (tmp_path / "RF.xmf").read_text()
    assert x.count("<Grid Name=\"Proc_") == 12 and 'Precision="4"' in x
    assert "./RF.h5:/sample_1_p11" in x


def test_one_file_per_tile(tmp_path):
    s, lay = _deck()
    f = _field(lay, np.float64, 5)
    S.write_sample_h5(None, tmp_path, "RF", f, s, lay, one_file=False, one_hdf_ds=False,
                      times=[1.0], time_labels=["Generation"])
    Np = [int(v) for v in lay["Np"]]
    for r in range(4):
        p = tmp_path / ("RF_proc_%05d.h5" % r)
        h = H5(p)
        assert [e[0] for e in h.entries] == ["sample_1_p%d" % r, "time_labels", "times"]
        g = S.tile_geometry(lay, (0, 0, 0), r)
        o = np.asarray(g["pos_0"]) - 1
        got = S.h5_read_dataset(p, "sample_1_p%d" % r)
        np.testing.assert_array_equal(got, f[o[0]:o[0] + Np[0], o[1]:o[1] + Np[1], o[2]:o[2] + Np[2]])
        assert (tmp_path / ("RF_proc_%05d.xmf" % r)).exists()
    assert "RF_proc_00003.h5:/sample_1_p3" in (tmp_path / "RF.xmf").read_text()


def test_reader_errors(tmp_path):
    p = tmp_path / "x.h5"
    p.write_bytes(b"not an hdf5 file" * 10)
    with pytest.raises(S.ScarlError):
        S.h5_list(p)
    s, lay = _deck()
    S.write_sample_h5(None, tmp_path, "RF", _field(lay), s, lay)
    with pytest.raises(S.ScarlError):
        S.h5_read_dataset(tmp_path / "RF.h5", "nothing")
    with pytest.raises(S.ScarlError):
        S.h5_read_attr(tmp_path / "RF.h5", "nothing")


def test_constant_field_file(tmp_path):
    S.write_constant_field_h5(tmp_path, "C", (0, 1, 2), (10, 11, 12), 3.5)
    h = H5(tmp_path / "C.h5")
    data, dims, attrs = h.dataset("samples")
    assert dims == (2, 2, 2) and np.all(data == 3.5)
    np.testing.assert_array_equal(attrs["xMax"], [10, 11, 12])
    ra = h.root_attrs
    assert [int(ra[k][0]) for k in ("method", "seedStart", "corrMod", "margiFirst")] == [-1] * 4
    np.testing.assert_array_equal(ra["xStep"], [10, 10, 10])
    np.testing.assert_array_equal(ra["corrL"], [-1, -1, -1])
    np.testing.assert_array_equal(ra["L"], [2, 2, 2])
    assert (tmp_path / "C.xmf").exists()


def test_overwrite_dataset_in_place(tmp_path):
    s, lay = _deck()
    S.write_sample_h5(None, tmp_path, "RF", _field(lay), s, lay, times=[0.0, 0.0],
                      time_labels=["Generation", "Write_file"])
    p = tmp_path / "RF.h5"
    size = os.path.getsize(p)
    S.h5_overwrite_dataset(p, "times", np.array([1.5, 2.5]))
    assert os.path.getsize(p) == size
    np.testing.assert_array_equal(H5(p).dataset("times")[0].ravel(), [1.5, 2.5])
    with pytest.raises(S.ScarlError):
        S.h5_overwrite_dataset(p, "times", np.zeros(3))


def test_stat_job_list_parsing():
    from scarl_b200 import stat
    corr, delete, files = stat.parse_jobs('2\n1\n0\n"./a/RF.h5"\nsamples\nb.h5\n"samples"\n')
    assert corr and not delete
    assert files == [("./a/RF.h5", "samples"), ("b.h5", "samples")]
