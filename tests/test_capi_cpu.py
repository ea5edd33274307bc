"""CPU-only checks of the boundary: the library loads, exports every symbol the
header declares, and refuses to run without a B200 (no CPU fallback)."""
import ctypes as C
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "cudamonsel_b200.h")
LIB = os.path.join(ROOT, "cudamonsel_b200", "libcudamonsel_b200.so")


def declared():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(cm_[a-z0-9_]+)\s*\(", text)))


def test_header_matches_binding_list():
    from cudamonsel_b200 import capi
    assert set(declared()) == set(capi.EXPORTS)


@pytest.mark.skipif(not os.path.exists(LIB), reason="library not built (run __graft_entry__.build())")
def test_library_exports_every_declared_symbol():
    lib = C.CDLL(LIB)
    missing = [s for s in declared() if not hasattr(lib, s)]
    assert not missing, missing


@pytest.mark.skipif(not os.path.exists(LIB), reason="library not built")
def test_fails_loudly_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from cudamonsel_b200 import capi
    with pytest.raises(capi.CMError):
        capi.Engine(0)


def test_scene_spec_replay_shapes():
    """The scene recorder produces the same call sequence the reference driver makes."""
    from cudamonsel_b200 import scenes
    sc = scenes.lines(nlines=3)
    names = [op for op, _ in sc.spec.ops]
    assert names.count("line") == 3 and names.count("translate") == 3
    assert names.count("region") == 5
    assert sc.spec.elements == {1, 6, 8, 14}


def test_yields_histogram_convention():
    """SE = counts(0..4) of 10 eV bins (values <= 40 eV with Histogram::bin's insertion-point
    rule), BSE = all back counts / N - SE (LinesOnLayers.cu:366-376)."""
    import numpy as np
    from cudamonsel_b200 import scenes
    back = np.zeros(102, dtype=np.int64)
    back[1:6] = [1, 2, 3, 4, 5]  # counts(0..4)
    back[6] = 7                  # counts(5): 40-50 eV, not SE
    back[101] = 3                # overflow (E == E0)
    bse, se = scenes.yields(back, 10, 1000.0, 100)
    assert abs(se[0] - 1.5) < 1e-7
    assert abs(bse[0] - (25 / 10 - 1.5)) < 1e-7


def test_scan_output_format(tmp_path):
    """The scan read-out writes LinesOnLayers' output.txt layout (std::to_string numbers) and PGM images."""
    import numpy as np
    from cudamonsel_b200 import scan
    assert scan.to_string(500.0) == "500.000000" and scan.to_string(3) == "3"
    txt = scan.output_text([(500.0, -1.5, 0.0, 0.1245, 2.335)], ["# Trajectories at each landing position: 100"],
                           12.5)
    assert txt == ("\n# Trajectories at each landing position: 100\n\nbeamE (eV)\tx(nm)\ty (nm)\tBSE yield\tSE yield"
                   "\n500.000000 -1.500000 0.000000 0.124500 2.335000\n12.500000")
    # yields from a histogram: 10 eV bins of a 500 eV beam, SE = bins below 50 eV
    back = np.zeros((1, 52), dtype=np.int64)
    back[0, 1:6] = 10     # 50 SE (bins 0..4)
    back[0, 30] = 20      # 20 BSE
    rows = scan.scan_rows(back, [[1e-9, 2e-9, -120e-9]], 500.0, 100, 50)
    assert abs(rows[0][3] - 0.2) < 1e-6 and abs(rows[0][4] - 0.5) < 1e-6 and abs(rows[0][1] - 1.0) < 1e-9
    img = np.arange(12, dtype=float).reshape(3, 4)
    scan.write_pgm(tmp_path / "a.pgm", img)
    g = scan.read_pgm(tmp_path / "a.pgm")
    assert g.shape == (3, 4) and g[0, 0] == 0 and g[2, 3] == 255
