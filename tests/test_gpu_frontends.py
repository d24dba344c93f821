"""The deck -> field -> HDF5 program (driver.run) and the Stat_ScaRL front
end (stat.main) end to end on the GPU."""
import io
import os

import numpy as np
import pytest

import scarl_b200 as S
from scarl_b200 import driver, stat

from test_h5 import H5

pytestmark = pytest.mark.gpu

CONFIG = """#Generation method (1 = FFT)
{gm}
#Create information file
0
#Delete sample in the end (0 = false, 1 = true)
0
#One File (0 = false, 1 = true)
{one_file}
#One hdf5 dataset (0 = false, 1 = true)
{one_ds}
#Input file name
"./input_ScaRL.txt"
"""

DECK = """"RESULTS"       #Output Folder
2               #Number of Samples
"S1"
0d0 0d0 0d0
15d0 12d0 9d0
3d0 2d0 3d0
1d0 1d0 1d0
4 4 4
1
2
1d0
0.3d0
5
"CONST"
0d0 0d0 0d0
1d0 1d0 1d0
1d0 1d0 1d0
1d0 1d0 1d0
5 5 5
1
1
2.5d0
0d0
1
"""


def _deck(tmp_path, gm=1, one_file=1, one_ds=1):
    (tmp_path / "config_ScaRL.txt").write_text(CONFIG.format(gm=gm, one_file=one_file, one_ds=one_ds))
    (tmp_path / "input_ScaRL.txt").write_text(DECK)


@pytest.mark.parametrize("one_file,one_ds", [(1, 1), (1, 0), (0, 0)])
def test_driver_writes_the_deck_samples(ctx, tmp_path, one_file, one_ds):
    _deck(tmp_path, 1, one_file, one_ds)
    done = driver.run(workdir=str(tmp_path), ctx=ctx, nb_procs=4)
    assert [d["name"] for d in done] == ["S1", "CONST"] and done[1]["constant"]
    res = tmp_path / "RESULTS"
    folder, samples = S.read_input_ScaRL(tmp_path / "input_ScaRL.txt")
    ref, lay = S.generate_sample(ctx, samples[0], generator=S.GEN_DCT, dtype=S.F64, nb_procs=4)
    if one_file and one_ds:
        got = S.h5_read_dataset(res / "S1.h5", "samples")
        np.testing.assert_array_equal(got, ref)
        h = H5(res / "S1.h5")
        t, dims, _ = h.dataset("times")
        assert dims == (1, 5) and np.all(t > 0)
        lab, _, _ = h.dataset("time_labels")
        assert lab.split() == [b"Read_input", b"Topology", b"Generation", b"Write_file",
                               b"Total_Wall_time"]
    elif one_file:
        for r in range(4):
            g = S.tile_geometry(lay, samples[0].xMinGlob[:], r)
            o = np.asarray(g["pos_0"]) - 1
            n = lay["Np"]
            got = S.h5_read_dataset(res / "S1.h5", "sample_1_p%d" % r)
            np.testing.assert_array_equal(got, ref[o[0]:o[0] + n[0], o[1]:o[1] + n[1], o[2]:o[2] + n[2]])
    else:
        assert all((res / ("S1_proc_%05d.h5" % r)).exists() for r in range(4))
    assert (res / "S1.xmf").exists() and (res / "CONST.h5").exists()
    # a second run keeps the first files and writes date-stamped ones
    done2 = driver.run(workdir=str(tmp_path), ctx=ctx, nb_procs=4)
    assert done2[0]["stem"].startswith("S1-")


def test_driver_fft_mpi_global_field(ctx, tmp_path):
    _deck(tmp_path, gm=2)
    done = driver.run(workdir=str(tmp_path), ctx=ctx, nb_procs=3)
    h = H5(tmp_path / "RESULTS" / "S1.h5")
    data, dims, attrs = h.dataset("samples")
    lay = done[0]["layout"]
    assert dims == tuple(int(v) for v in lay["L"][::-1])
    assert list(h.root_attrs["nb_procs"]) == [1]


def test_stat_front_end(ctx, tmp_path):
    _deck(tmp_path)
    driver.run(workdir=str(tmp_path), ctx=ctx, nb_procs=4)
    path = str(tmp_path / "RESULTS" / "S1.h5")
    field = S.h5_read_dataset(path, "samples")
    out = io.StringIO()
    res = stat.main(io.StringIO(f"1\n1\n0\n{path}\nsamples\n"), ctx=ctx, out=out)
    _, avg, std, cl = res[0]
    assert avg == pytest.approx(field.mean(), rel=1e-12)
    assert std == pytest.approx(field.std(), rel=1e-10)
    L = list(field.shape)
    sk = S.rebuild_Sk(ctx, field, L, avg, std)
    xs = S.h5_read_attr(path, "xStep")
    np.testing.assert_allclose(cl, S.rebuild_corrL(sk, L, xs), rtol=1e-12)
    # statistics added to the result file (a new root header), data intact
    h = H5(path)
    assert h.root_attrs["globalAvg"][0] == pytest.approx(avg, rel=1e-15)
    np.testing.assert_allclose(h.root_attrs["corrL_out"], cl, rtol=1e-15)
    assert len(h.root_attrs["Sk_1"]) == L[0] // 2
    np.testing.assert_array_equal(S.h5_read_dataset(path, "samples"), field)
    assert h.eof == os.path.getsize(path)
    st = H5(tmp_path / "RESULTS" / "STAT_S1.h5")
    assert st.entries == [] and st.root_attrs["old_file_mb_size"][0] > 0
    for k in ("Np", "L", "xStep", "corrL", "globalStdDev", "Sk_3"):
        assert k in st.root_attrs
    # a second pass replaces the statistics instead of duplicating them
    stat.main(io.StringIO(f"1\n1\n0\n{path}\nsamples\n"), ctx=ctx, out=io.StringIO())
    names = [m[8:8 + int.from_bytes(m[2:4], "little") - 1] for t, m in H5(path).root_msgs if t == 0xC]
    assert names.count(b"globalAvg") == 1 and names.count(b"Sk_2") == 1
    # deleteSampleInTheEnd removes the sample's files, not the statistics
    stat.main(io.StringIO(f"1\n0\n1\n{path}\nsamples\n"), ctx=ctx, out=io.StringIO())
    assert not os.path.exists(path) and not (tmp_path / "RESULTS" / "S1.xmf").exists()
    assert (tmp_path / "RESULTS" / "STAT_S1.h5").exists()
