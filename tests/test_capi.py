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
