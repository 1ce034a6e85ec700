"""Checkpoint / resume of the Darcy and fluid ``run`` loops against the
reference's semantics (``src/base.py:82-87,869-928``): a checkpoint holds the
populations after step k, only the latest is kept, a resumed run continues at
step k + 1 and must end bit-identical to an uninterrupted run, and resuming
when ``t_max`` does not exceed k + 1 raises ``ValueError``."""
import os

import numpy as np
import pytest
import torch

from problems import make_cavity, make_darcy

pytestmark = pytest.mark.gpu


def _darcy(G, **kw):
    return make_darcy(G, "anti")(lattice=G.LatticeD2Q9("f64/f64"), omega=1.25, nx=20, ny=16, nz=0,
                                 precision="f64/f64", print_info_rate=0, **kw)


def _cavity(G, **kw):
    C, om = make_cavity(G, "bgk")
    return C(lattice=G.LatticeD2Q9("f64/f64"), omega=om(24), nx=24, ny=24, nz=0, precision="f64/f64",
             print_info_rate=0, **kw)


@pytest.mark.parametrize("make", [_darcy, _cavity], ids=["darcy", "fluid"])
def test_resume_matches_uninterrupted_run(tmp_path, make):
    import xlb_biot_b200.api as G
    ck = str(tmp_path / "ck")
    ref = make(G).run(10)
    first = make(G, checkpoint_rate=3, checkpoint_dir=ck)
    first.run(7)
    assert sorted(os.listdir(ck)) == ["checkpoint_00000006.pt"]          # max_to_keep = 1
    resumed = make(G, checkpoint_rate=3, checkpoint_dir=ck, restore_checkpoint=True).run(10)
    torch.cuda.synchronize()
    assert np.array_equal(resumed.cpu().numpy(), ref.cpu().numpy())


def test_resume_past_t_max_raises(tmp_path):
    import xlb_biot_b200.api as G
    ck = str(tmp_path / "ck")
    _cavity(G, checkpoint_rate=3, checkpoint_dir=ck).run(6)
    with pytest.raises(ValueError, match="exceeded maximum allowable steps"):
        _cavity(G, checkpoint_rate=3, checkpoint_dir=ck, restore_checkpoint=True).run(7)
