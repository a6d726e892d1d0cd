"""The bench's byte model covers every kernel the fused step launches: each
profiled launch label of csrc/pfag_fused_impl.cuh has an algorithmic-bytes
entry in bench.kernel_bytes, except the few-warp reductions, whose bytes are a
few KB and which the roofline does not rate."""
import os
import re

import bench
from multicellular_phase_field_active_gel_organoids_b200.params import CONFIGS

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REDUCTIONS = {"kf_area_tiles", "kfl_sum_ecm", "kl_decide", "kl_copy", "kf_rho_ring"}


def labels():
    src = open(os.path.join(ROOT, "multicellular_phase_field_active_gel_organoids_b200", "csrc",
                            "pfag_fused_impl.cuh")).read()
    out = set()
    for m in re.finditer(r'pfag_prof_begin\(c, ([^;]*)\);', src):
        out.update(re.findall(r'"(k[a-z_0-9A-Z]+)"', m.group(1)))
    return out


def test_every_launch_label_has_bytes():
    names = labels()
    assert {"kr_boxA", "kbl_rowsD1", "kl_relax_tma", "kf_update_rows"} <= names
    cfg = CONFIGS["cfg1"]()
    kb = bench.kernel_bytes(cfg, 32, {"cell_iters_sum": cfg.ncells, "lum_iters": 1, "ecm_iters": 2}, 10 ** 6,
                            10 ** 6)
    missing = sorted(n for n in names - REDUCTIONS if n not in kb)
    assert not missing, missing
    assert all(kb[n] > 0 for n in names - REDUCTIONS)
