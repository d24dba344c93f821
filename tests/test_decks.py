"""Deck readers (SRC_F/read_input.f90) on the reference's own decks and on
list-directed edge cases."""
import os

import numpy as np
import pytest

import scarl_b200 as S

DECKS = os.path.join(os.path.dirname(__file__), "golden", "decks")


def test_config_3_test():
    c = S.read_config_ScaRL(os.path.join(DECKS, "3_TEST", "config_ScaRL.txt"))
    assert c == dict(gen_meth=1, c_info_file=True, d_sample=False, one_file=True, one_hdf_ds=True,
                     input_file="./input_ScaRL.txt")


def test_config_fusion_inline_comments():
    c = S.read_config_ScaRL(os.path.join(DECKS, "testFusion", "config_ScaRL.txt"))
    assert c["gen_meth"] == 2 and c["c_info_file"] and not c["d_sample"]
    assert c["input_file"] == "./input_ScaRL.txt"


def test_config_defaults_when_missing(tmp_path):
    c = S.read_config_ScaRL(tmp_path / "nope.txt")
    assert c == dict(gen_meth=1, c_info_file=False, d_sample=False, one_file=True,
                     one_hdf_ds=True, input_file="./input_ScaRL.txt")


def test_input_3_test():
    folder, samples = S.read_input_ScaRL(os.path.join(DECKS, "3_TEST", "input_ScaRL.txt"))
    # the deck declares one sample; its second block is never read
    assert folder == "SAMPLES" and len(samples) == 1
    a = S.sample_dict(samples[0])
    assert a["name"] == "Sample_Test_1"
    assert a["xMinGlob"] == [0, 0, 0] and a["xMaxGlob"] == [10, 10, 10]
    assert a["corrL"] == [1, 1, 1] and a["overlap"] == [1, 1, 1]
    assert a["pointsPerCorrL"] == [5, 5, 5]
    assert (a["corrMod"], a["margiFirst"], a["avg"], a["std_dev"], a["seedBase"]) == (1, 2, 1.0, 1.0, 1)


def test_input_second_sample_when_declared(tmp_path):
    txt = open(os.path.join(DECKS, "3_TEST", "input_ScaRL.txt")).read()
    deck = tmp_path / "in.txt"
    deck.write_text(txt.replace("1               #Number of Samples", "2 #Number of Samples"))
    _, samples = S.read_input_ScaRL(deck)
    b = S.sample_dict(samples[1])
    assert b["name"] == "sample_2" and b["xMaxGlob"] == [20, 20, 20]
    assert b["overlap"] == [5, 5, 5] and b["seedBase"] == 20


def test_input_fusion():
    folder, samples = S.read_input_ScaRL(os.path.join(DECKS, "testFusion", "input_ScaRL.txt"))
    s = S.sample_dict(samples[0])
    assert s["name"] == "BASIC_Sample" and s["xMaxGlob"] == [30, 30, 30] and s["margiFirst"] == 1


def test_extra_config():
    found, topo = S.read_extra_config_ScaRL(os.path.join(DECKS, "GENERAL_BASH", "extra_config_ScaRL.txt"))
    assert found and list(topo) == [2, 2, 2]
    found, topo = S.read_extra_config_ScaRL(os.path.join(DECKS, "nothing_here.txt"))
    assert not found and list(topo) == [-1, -1, -1]


def test_sem_mode():
    folder, samples = S.read_input_SEM(os.path.join(DECKS, "SEM_TEST"))
    assert folder == "./mat/h5" and len(samples) == 6
    d = [S.sample_dict(s) for s in samples]
    assert [x["name"] for x in d] == ["Mat_25_Kappa", "Mat_25_Mu", "Mat_25_Density",
                                      "Mat_26_Kappa", "Mat_26_Mu", "Mat_26_Density"]
    rho, vp, vs = 2200.0, 3553.0, 2175.0
    assert d[0]["avg"] == rho * (vp * vp - 4.0 * (vs * vs) / 3.0)
    assert d[1]["avg"] == rho * (vs * vs) and d[2]["avg"] == rho
    assert d[0]["std_dev"] == 0.5 * d[0]["avg"] and d[2]["std_dev"] == 0.0
    # the material number is the first column of domains.txt (read_input.f90:478)
    assert d[0]["xMinGlob"] == [4500.0, 4500.0, 9500.0]
    assert d[0]["xMaxGlob"] == [14700.0, 14505.0, 14720.0]
    assert d[3]["xMinGlob"] == [9500.0, 9467.8285, 14500.0]
    assert all(x["overlap"] == [5, 5, 5] and x["pointsPerCorrL"] == [5, 5, 5] for x in d)
    assert [x["seedBase"] for x in d] == [1, 2, 3, 1, 2, 3]


def test_list_directed_forms(tmp_path):
    deck = tmp_path / "in.txt"
    deck.write_text("""  # leading comment
'OUT dir'   ! trailing text
1
#--
"name, with comma"
-1.5D0,2*0d0
3*1.25e1
1d0 2.5D-1 1q0 / ignored
2.0 2.0 2.0
7 8 9
2
1
1.5
0.25
-3
""")
    folder, samples = S.read_input_ScaRL(deck)
    s = S.sample_dict(samples[0])
    assert folder == "OUT dir" and s["name"] == "name, with comma"
    assert s["xMinGlob"] == [-1.5, 0.0, 0.0] and s["xMaxGlob"] == [12.5] * 3
    assert s["corrL"] == [1.0, 0.25, 1.0]
    assert s["pointsPerCorrL"] == [7, 8, 9] and s["corrMod"] == 2 and s["seedBase"] == -3


def test_truncated_deck_is_an_io_error(tmp_path):
    deck = tmp_path / "in.txt"
    deck.write_text('"x"\n2\n"a"\n0 0 0\n')
    with pytest.raises(S.ScarlError) as e:
        S.read_input_ScaRL(deck)
    assert e.value.code == 6
    with pytest.raises(S.ScarlError):
        S.read_input_ScaRL(tmp_path / "missing.txt")


def test_deck_samples_layout_runs(oracle):
    _, samples = S.read_input_ScaRL(os.path.join(DECKS, "3_TEST", "input_ScaRL.txt"))
    for s in samples:
        S.verify_inputs(s)
        d = S.sample_dict(s)
        got = S.sample_layout(s, 1, 8)
        ref = oracle.sample_layout(d["xMinGlob"], d["xMaxGlob"], d["corrL"], d["overlap"],
                                   d["pointsPerCorrL"], 1, 8)
        np.testing.assert_array_equal(got["Np"], ref["Np"])
