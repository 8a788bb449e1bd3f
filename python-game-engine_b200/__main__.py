"""``python python-game-engine_b200 {run,validate,list} ...``: the cfd-bench command line on
the CUDA backend (benchmarking.main). The package directory is not an identifier, so the
package is imported by name from its parent directory."""
import importlib
import os
import sys

if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    importlib.import_module("python-game-engine_b200")
    sys.exit(importlib.import_module("python-game-engine_b200.benchmarking").main(sys.argv[1:]))
