"""Drop-in replay: the exact calls the reference's own runner makes to ``propagate_logD``.

``tests/golden/make_golden.py dropin`` ran the unmodified reference ``ticc.solve`` with the
name ``propagate_logD`` in ``pyticc.propagation.runner`` (the call at runner.py:293) wrapped
to record every call's arguments and result, over a radial grid split into several windows.
Here those same arguments go to this library's ``propagate_logD`` in the same order, the
result of one call feeding the next as the reference's runner chains them, and the final
Y goes through this library's BF -> SF transform and ``get_Smat``.  Tolerances: Y per call
within 1e-10 of its largest entry; S within 1e-8.
"""

from __future__ import annotations

import numpy as np
import pytest

import pyticc_b200 as tb
from pyticc_b200.propagation.logd import propagate_logD
from tests.conftest import load_golden

pytestmark = pytest.mark.gpu


def test_replayed_reference_calls_give_the_reference_results():
    data, params = load_golden("dropin_calls")
    assert params["n_calls"] >= 2
    Y = None
    for i in range(params["n_calls"]):
        args = {k: data[f"call{i}_{k}"] for k in ("Y_initial", "total_energies", "radial_half_steps", "W_base_start", "W_base_mid", "W_base_end")}
        # the reference's own input for this call and, after the first, the chained one
        own = propagate_logD(args["Y_initial"], args["total_energies"], float(data[f"call{i}_reduced_mass"]), args["radial_half_steps"], args["W_base_start"], args["W_base_mid"], args["W_base_end"])
        want = data[f"call{i}_Y_final"]
        np.testing.assert_allclose(own.cpu().numpy(), want, rtol=0, atol=1e-10 * np.abs(want).max())
        if Y is not None:
            np.testing.assert_allclose(Y.cpu().numpy(), args["Y_initial"], rtol=0, atol=1e-10 * np.abs(args["Y_initial"]).max())
        Y = propagate_logD(args["Y_initial"] if Y is None else Y, args["total_energies"], float(data[f"call{i}_reduced_mass"]), args["radial_half_steps"], args["W_base_start"], args["W_base_mid"], args["W_base_end"])
    Y_sf = tb.transform_logD_BF_to_SF(Y, data["Bmat"])
    smats = tb.get_Smat(Y_sf, float(data["Rmatch"]), data["energies"], float(data["call0_reduced_mass"]), data["E_int"], data["L"])
    for e, S in enumerate(smats):
        k = int(data["n_open"][e])
        assert S.shape == (k, k)
        if k:
            assert np.abs(np.asarray(S) - data["Smat"][e, :k, :k]).max() <= 1e-8

