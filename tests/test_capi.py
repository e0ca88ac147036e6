"""The C ABI library loads and exports every function include/sinksim_b200.h declares; entry points that need a
device report SSB_ENODEVICE cleanly on a machine without one; host-side entry points work without a GPU."""
import ctypes as C
import os
import re

import pytest

import sinksim_b200 as ssb
from _support import ROOT, titanic


def declared_functions():
    text = open(os.path.join(ROOT, "include", "sinksim_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?(?:int|void|double|const char\*|char\*)\s*\*?\s*(ssb_\w+)\s*\(", text, flags=re.M)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("ssb_batch_create", "ssb_batch_run", "ssb_batch_set_connection_area", "ssb_run_sweep", "ssb_compare_results"):
        assert must in names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(ssb.library_path())
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_error_plumbing():
    assert ssb.lib().ssb_version().decode().startswith("sinksim-b200")
    with pytest.raises(ssb.SinksimError):
        ssb.Batch("/nonexistent/ship.json", "/nonexistent/sim.json", numerics="oracle")


def test_no_device_is_reported_not_faked():
    ok, why = ssb.available()
    if ok:
        pytest.skip("a CUDA device is present")
    ship, sim = titanic()
    with pytest.raises(ssb.SinksimError) as e:
        ssb.Batch(ship, sim, count=2, numerics="portable")
    assert e.value.code == -5


def test_compare_results_on_host(tmp_path):
    """The exact comparison of batch-results (sinksim_sweep --compare) runs on the host."""
    doc = ('{"format":"sinksim.batch-results","formatVersion":1,"ship":"s","sim":"m","numerics":"portable","engine":"e","tMax":10,"every":5,'
           '"instances":[{"id":"a","foundered":false,"founderT":-1,"tEnd":10,"steps":40,"final":{"trimDeg":0.5,"listDeg":0,"waterT":1,'
           '"draftF":2,"draftA":3,"inflowTpm":0},"events":[],"curve":{"t":[0,5,10],"trim":[0,0.25,0.5],"list":[0,0,0],"water":[0,0.5,1],'
           '"inflow":[0,0,0],"draftF":[2,2,2],"draftA":[3,3,3]}}]}')
    a = tmp_path / "a.json"
    b = tmp_path / "b.json"
    a.write_text(doc)
    b.write_text(doc.replace('"trim":[0,0.25,0.5]', '"trim":[0,0.25,0.5000000000000001]'))
    assert ssb.compare_results(str(a), str(a))[1] == 0
    compared, differing, first = ssb.compare_results(str(a), str(b))
    assert differing == 1 and "curve[2] trim" in first


def test_launch_plan_orders_only_phases_after_the_first():
    """The kernels a run captures: the claim-order pair never precedes the first phase (it ranks what the phase before
    left unfinished), with or without a caller's first-phase order, which adds no kernel."""
    plan = ssb.launch_plan([512, 64, 0])
    assert plan == [("start_run", -1), ("phase", 0), ("claim_order", 1), ("phase", 1), ("claim_order", 2), ("phase", 2)]
    # one phase only: nothing to rank
    assert ssb.launch_plan([0]) == [("start_run", -1), ("phase", 0)]
    # claim by index, or bounded launches (which the host drives round by round): no ranking kernels
    assert ssb.launch_plan([512, 0], claim_by_index=True) == [("start_run", -1), ("phase", 0), ("phase", 1)]
    assert ssb.launch_plan([512, 0], steps_per_launch=2000) == [("start_run", -1), ("phase", 0), ("phase", 1)]
    # a hand-over bound beyond what the ranking kernel takes: claim by index
    assert ssb.launch_plan([100000, 0]) == [("start_run", -1), ("phase", 0), ("phase", 1)]


def test_launch_plan_refuses_a_short_buffer():
    o = ssb._Options()
    ssb.lib().ssb_batch_options_init(C.byref(o))
    y = (C.c_int32 * 3)(512, 64, 0)
    kinds = (C.c_int32 * 2)()
    n = C.c_int32()
    rc = ssb.lib().ssb_launch_plan(C.byref(o), 3, y, kinds, None, 2, C.byref(n))
    assert rc == -1 and n.value == 6
