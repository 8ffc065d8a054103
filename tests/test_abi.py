"""CPU-side checks of the C-ABI library: it loads, exports every entry point
``include/*.h`` declares, and its host logic (contract checks, hot start,
bond probability, seed folding) agrees with the oracle.  No device calls."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

import plaquette_b200 as plq

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names |= set(re.findall(r"\b(plq_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(plq.LIB_PATH)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    assert len(declared_symbols()) >= 20


def test_python_binding_covers_the_header():
    plq.lib()
    import plaquette_b200.ensemble  # noqa: F401  (registers its signatures)
    import plaquette_b200.serving  # noqa: F401
    import plaquette_b200.slabs  # noqa: F401
    assert set(declared_symbols()) <= set(plq.exported_symbols())


def test_version_and_strerror():
    assert "sm_100a" in plq.version()
    assert plq.lib().plq_strerror(plq.PLQ_ECAP).decode().startswith("cluster labeling")


def _desc(**kw):
    base = dict(beta=0.44, seed=1)
    base.update(kw)
    model = base.pop("model", plq.ISING)
    q = base.pop("q", 2)
    shape = base.pop("shape", (4, 4))
    upd = base.pop("updater", plq.METROPOLIS)
    return plq.make_desc(model, q, shape, upd, **base)


def test_even_extents_message_matches_reference():
    # src/device.rs:714-719
    with pytest.raises(plq.ContractError, match=r"the parallel site checkerboard needs even lattice extents, got \[3, 4\]"):
        plq.validate(_desc(shape=(3, 4)))
    with pytest.raises(plq.ContractError, match=r"the parallel link checkerboard needs even lattice extents, got \[4, 5\]"):
        plq.validate(_desc(model=plq.GAUGE, shape=(4, 5)))


def test_cluster_contracts_match_reference():
    # src/updater.rs:447-483
    with pytest.raises(plq.ContractError, match="invariant under relabeling"):
        plq.validate(_desc(updater=plq.CLUSTER, h=0.5))
    with pytest.raises(plq.ContractError, match="two-cycle"):
        plq.validate(_desc(updater=plq.CLUSTER, extent=plq.EXTENT_ALL, relabel=plq.RELABEL_FORCED))
    with pytest.raises(plq.ContractError, match="non-negative gap, got -2"):
        plq.validate(_desc(updater=plq.CLUSTER, j=-1.0))
    with pytest.raises(plq.ContractError, match="site field"):
        plq.validate(_desc(model=plq.GAUGE, updater=plq.CLUSTER))
    # odd extents are fine for a cluster chain (gpu_cluster.rs:52-53)
    plq.validate(_desc(updater=plq.CLUSTER, shape=(5, 3)))


def test_other_contracts():
    with pytest.raises(plq.ContractError, match="batch size must be positive"):
        plq.validate(_desc(batch=0))
    with pytest.raises(plq.ContractError, match="at least two dimensions"):
        plq.validate(_desc(model=plq.GAUGE, shape=(4,)))
    with pytest.raises(plq.ContractError, match="at least two states"):
        plq.validate(_desc(model=plq.POTTS, q=1))
    # Potts Metropolis at q >= 3 on the PCG stream is valid (the sequential walk)
    plq.validate(_desc(model=plq.POTTS, q=3, rng=plq.RNG_STREAM))


@pytest.mark.parametrize("seed,q,n", [(20260718, 2, 4096), (7, 3, 5000), (1, 5, 777)])
def test_hot_start_matches_oracle(oracle, seed, q, n):
    got, draws = plq.hot_start(seed, q, n)
    rng = oracle.PcgStream(seed)
    want = oracle.hot_start(n, q, rng)
    assert np.array_equal(got, want)
    assert draws == rng.draws


def test_bond_probability_and_fold_seed(oracle):
    for beta in (0.0, 0.2216544, 0.4406868, 3.0):
        assert plq.bond_probability(plq.ISING, 1.0, beta) == oracle.Model.ising(1.0).bond_probability(beta)
        assert plq.bond_probability(plq.POTTS, 0.7, beta) == oracle.Model.potts(3, 0.7).bond_probability(beta)
    for s in (0, 1, 2**40 + 5, 20260718):
        assert plq.fold_seed(s) == oracle.fold_seed(s)


def test_no_device_here_is_none_or_context():
    # Gpu::new() is None without a device (src/device.rs:42-44)
    g = plq.Gpu.new()
    if plq.device_count() == 0:
        assert g is None


def test_descriptor_layout_matches_the_header(tmp_path):
    """The ctypes descriptor has the C struct's size and field offsets
    (gcc on include/plaquette.h)."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    fields = [f[0] for f in plq.ChainDesc._fields_]
    src = tmp_path / "layout.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "plaquette.h"', "int main(void) {",
             '  printf("%zu\\n", sizeof(plq_chain_desc));']
    lines += [f'  printf("%zu\\n", offsetof(plq_chain_desc, {f}));' for f in fields]
    lines += ["  return 0;", "}"]
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert got[0] == C.sizeof(plq.ChainDesc)
    assert got[1:] == [getattr(plq.ChainDesc, f).offset for f in fields]


def test_integration_binding_lists_every_entry_point():
    """The Rust extern block a maintainer would add names every entry point
    of the header."""
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    block = text[text.index('extern "C" {'):]
    block = block[:block.index("\n}\n")]
    bound = set(re.findall(r"pub fn (plq_[a-z0-9_]+)\(", block))
    assert set(declared_symbols()) <= bound, sorted(set(declared_symbols()) - bound)


def test_python_constants_mirror_the_header():
    """The ctypes layer's status codes, descriptor flags and limits equal the
    header's #defines (a flag added to one side only would silently select
    another pass body)."""
    text = open(os.path.join(ROOT, "include", "plaquette.h")).read()
    defines = {m.group(1): int(m.group(2)) for m in re.finditer(r"^#define (PLQ_[A-Z0-9_]+) (\d+)", text, re.M)}
    codes = ["PLQ_OK", "PLQ_ENODEV", "PLQ_EINVAL", "PLQ_EUNSUPPORTED", "PLQ_ECUDA", "PLQ_ENOMEM", "PLQ_ECAP",
             "PLQ_EDEVICE", "PLQ_EBUSY"]
    for name in codes:
        assert getattr(plq, name) == defines[name], name
    flags = [n for n in defines if n.startswith("PLQ_FLAG_")]
    assert len(flags) >= 6
    for name in flags:
        assert getattr(plq, name[len("PLQ_"):]) == defines[name], name
    assert plq.MAX_D == defines["PLQ_MAX_D"] and plq.MAX_Q == defines["PLQ_MAX_Q"]
