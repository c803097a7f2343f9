"""Static checks on the host layer, the counterparts of the reference's
test/test_discipline.jl:11-45 (no synchronization inside a loop: a sweep may
not wait per panel) and test/test_api_surface.jl (a frozen export list, and
the host layers never name a vendor package). CPU only."""
import ast
import os

import pytest

from conftest import ROOT

PKG = os.path.join(ROOT, "funicular.jl_b200")
HOST_MODULES = ("device_api.py", "kernels.py", "plan.py", "panels.py", "executor.py", "panelblas.py", "ghosts.py",
                "autodiff.py", "autotune.py")
SYNCHRONIZATION = {"sync_all", "sync_queue", "sync_event"}


def syncs_inside_loops(tree) -> list[str]:
    """Names of synchronizing calls made inside a for/while loop, outside
    functions whose own name starts with `sync` (those may loop over queues)."""
    found = []

    def visit(node, inloop):
        if isinstance(node, (ast.FunctionDef, ast.AsyncFunctionDef)):
            if node.name.startswith("sync"):
                return
            inloop = False   # a function defined in a loop body runs when called
        if isinstance(node, ast.Lambda):
            inloop = False
        if inloop and isinstance(node, ast.Call):
            f = node.func
            name = f.attr if isinstance(f, ast.Attribute) else f.id if isinstance(f, ast.Name) else None
            if name in SYNCHRONIZATION:
                found.append(name)
        nested = inloop or isinstance(node, (ast.For, ast.While, ast.AsyncFor))
        for child in ast.iter_child_nodes(node):
            visit(child, nested)

    visit(tree, False)
    return found


def parse(name):
    with open(os.path.join(PKG, name)) as f:
        return ast.parse(f.read(), filename=name)


@pytest.mark.parametrize("module", HOST_MODULES)
def test_no_synchronization_inside_a_loop(module):
    assert syncs_inside_loops(parse(module)) == []


def test_the_loop_detector_has_teeth():
    assert syncs_inside_loops(ast.parse("def sweep(b, q):\n for j in range(3):\n  b.sync_queue(q)\n")) == ["sync_queue"]
    assert syncs_inside_loops(ast.parse("def sweep(b, q):\n for j in range(3):\n  pass\n b.sync_queue(q)\n")) == []
    assert syncs_inside_loops(ast.parse("def sync_all_queues(b, qs):\n for q in qs:\n  b.sync_queue(q)\n")) == []
    assert syncs_inside_loops(ast.parse("while True:\n sync_all()\n")) == ["sync_all"]


VENDOR = {"torch", "cupy", "numba", "triton", "cuda", "pycuda", "h5py", "tensorflow", "jax"}


@pytest.mark.parametrize("module", HOST_MODULES)
def test_host_layer_names_no_vendor_package(module):
    # The device is reached through the C ABI alone (_lib.py loads the
    # library); the host layers, like the reference's src/, import no vendor
    # package.
    for node in ast.walk(parse(module)):
        if isinstance(node, ast.Import):
            names = [a.name for a in node.names]
        elif isinstance(node, ast.ImportFrom):
            names = [node.module or ""]
        else:
            continue
        for name in names:
            assert name.split(".")[0] not in VENDOR, f"{module} imports {name}"


# The reference's exports (src/Funicular.jl:18-20) and where each one lives
# here; the ones outside the hot path are out of scope (the disk tier, the
# elementwise BLAS, the operator probes, the CPU backend).
REFERENCE_EXPORTS = {
    "CPUBackend": None, "ResidencyPlan": "ResidencyPlan", "PanelMatrix": "PanelMatrix", "GhostPanels": "GhostPanels",
    "npanels": "PanelMatrix.npanels", "panelwidth": "PanelMatrix.panelwidth", "panelrange": "PanelMatrix.panelrange",
    "copycols!": None, "foreachpanel": "foreachpanel", "check_operator": None, "gram": "gram",
    "panelmul!": "panelmul", "rightmul!": "rightmul", "cholqr2!": "cholqr2", "project": "project", "scale!": None,
    "save": None, "load": None,
}

# Feature-creep tripwire: the public surface is fixed, and adding to it
# means editing this list on purpose.
PUBLIC_API = sorted([
    "ArgumentError", "DimensionMismatch", "NotPositiveDefinite", "DeviceError", "OutOfDeviceMemory", "B200Backend",
    "DeviceMatrix", "HostSlab", "b200_backend", "kernels", "LIBRARY_PATH", "GiB", "ResidencyPlan",
    "choose_panel_width", "row_block_height", "device_bytes_allocated", "host_bytes_reserved", "host_bytes_in_use",
    "host_bytes_free", "PanelMatrix", "free", "sweep", "foreachpanel", "readpanels", "writepanels", "updatepanels",
    "PanelSteps", "RowSteps", "rowtraversal", "gram", "panelmul", "cholqr2", "cholqr3", "project", "rightmul",
    "DenseOperator", "ColumnOperator", "DeviceOperator", "Laplacian7", "HermitianBand", "cholesky_upper",
    "GhostPanels", "isghost", "autodiff", "rrule", "autotune",
])


def test_public_api_surface(fb):
    assert sorted(fb.__all__) == PUBLIC_API
    for name in fb.__all__:
        assert hasattr(fb, name), name


def test_every_reference_export_is_mirrored_or_out_of_scope(fb):
    for ref, ours in REFERENCE_EXPORTS.items():
        if ours is None:
            continue
        obj = fb
        for part in ours.split("."):
            obj = getattr(obj, part)
        assert callable(obj), ref


def test_exports_are_documented(fb):
    for name in fb.__all__:
        obj = getattr(fb, name)
        if callable(obj) or hasattr(obj, "__file__"):
            assert (getattr(obj, "__doc__", None) or "").strip(), f"{name} has no docstring"
