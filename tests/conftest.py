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
