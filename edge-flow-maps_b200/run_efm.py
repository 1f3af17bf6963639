"""Drop-in for the reference's run_efm.py driver: same CLI (-c/--case,
-n/--name) and loop, on the sm_100a library (see edgeb200/driver.py)."""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from edgeb200.driver import main  # noqa: E402

if __name__ == "__main__":
    main("efm")
