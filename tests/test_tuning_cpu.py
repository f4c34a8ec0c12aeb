"""The tuning tables committed beside the package hold only parameters the
library knows, within the ranges it accepts (csrc/rans_tuning.cu), and the
header documents every parameter."""

import glob
import json
import os

from conftest import ROOT

KNOWN = {
    "o1_four_max_streams": (-1, 1 << 30),
    "o1_top_latency_pct": (0, 100000),
    "o1_top_max": (-1, 1 << 30),
    "o1_top_exclusive": (0, 1),
    "o1_top_small_per_sm": (1, 4),
    "cta_cap_o0": (1, 64),
    "cta_cap_o1_small": (1, 64),
    "cta_cap_o1_wide": (1, 64),
    "cta_cap_o1_four": (1, 16),
    "cta_cap_o1_global": (1, 64),
    "cta_cap_o1_small_topped": (1, 64),
    "cta_cap_o1_wide_topped": (1, 64),
    "dense_edge_small": (0, 160 * 1024),
    "dense_edge_large": (0, 160 * 1024),
    "enc_run_ctas_per_sm": (1, 64),
    "enc_run_ctas_per_sm_uniform": (1, 64),
    "enc_o1_keys": (0, 1),
    "host_enc_chunks": (1, 16),
    "host_dec_chunks": (1, 16),
    "host_in_place": (-1, 1),
    "host_out_mirror": (0, 1),
}


def test_tuning_tables_hold_known_parameters():
    for path in glob.glob(os.path.join(ROOT, "fqxv_b200", "tuning", "*.json")):
        with open(path) as f:
            t = json.load(f)
        assert set(t["params"]) <= set(KNOWN), path
        for k, v in t["params"].items():
            lo, hi = KNOWN[k]
            assert isinstance(v, int) and lo <= v <= hi, (path, k, v)
        # the library's reader takes the first occurrence of a quoted name
        # anywhere in the file, so measurement keys must not repeat one
        text = open(path).read()
        for k in KNOWN:
            assert text.count('"%s"' % k) <= 1, (path, k)


def test_header_documents_every_parameter():
    text = open(os.path.join(ROOT, "include", "fqxv_rans_gpu.h")).read()
    for k in KNOWN:
        assert k in text, k
