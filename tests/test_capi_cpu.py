"""The C ABI library loads without a GPU and exports every entry point that
include/mgc.h declares."""
import os
import re

import mgbrain_b200 as mgb

HDR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "mgc.h")


def declared():
    txt = open(HDR).read()
    # declarations: a return type then the name directly followed by '('
    return sorted(set(re.findall(r"^[A-Za-z_][\w \*]*?\b(mgc_[a-z_]+)\(", txt, re.M)))


def test_library_exports_header_symbols():
    L = mgb.lib()
    names = declared()
    assert "mgc_create" in names and "mgc_run" in names
    for n in names:
        assert hasattr(L, n), n
    assert set(names) <= set(mgb.capi.EXPORTED)


def test_no_device_is_reported_not_fatal():
    import torch
    if torch.cuda.is_available():
        return
    import numpy as np
    try:
        mgb.Simulator.from_arrays(2, np.array([5, 5], np.int8), [0], [1], [0.1], [1],
                                  np.r_[0.0001, np.zeros(29)].astype(np.float32))
    except mgb.MgcError as e:
        assert e.status == mgb.capi.MGC_ERR_NODEVICE
    else:
        raise AssertionError("expected MgcError without a GPU")
