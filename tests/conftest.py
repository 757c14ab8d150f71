import os
import sys

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (REPO, os.path.join(REPO, "vqc.jl_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)
# spawned worker processes (multi-rank tests) import the package too
os.environ["PYTHONPATH"] = os.pathsep.join([REPO, os.path.join(REPO, "vqc.jl_b200"),
                                            os.environ.get("PYTHONPATH", "")])


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the sm_100a engine)")


try:
    import pytest

    @pytest.fixture(autouse=True)
    def _debug_index_checks(request):
        """With the debug library (VQC_DEBUG_LIB=1), every GPU test must leave
        no device access out of bounds: the index checks record and skip such
        an access, and this reads their records after the test."""
        if os.environ.get("VQC_DEBUG_LIB") != "1" or request.node.get_closest_marker("gpu") is None:
            yield
            return
        from vqcb200 import _lib
        assert _lib.load().vqc_debug_build() == 1
        _lib.debug_status(reset=True)
        yield
        hits, line, index, limit = _lib.debug_status(reset=True)
        assert hits == 0, "%d device accesses out of bounds; first at line %d: index %d, limit %d" % (
            hits, line, index, limit)
except ImportError:  # pragma: no cover
    pass
