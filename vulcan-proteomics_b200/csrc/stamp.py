"""Source hash of a native library (printed; the Makefile stores it next to the built .so and the loader refuses
a library whose stored hash differs from the sources it is loaded with)."""
import glob
import hashlib
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def sources(which: str) -> list[str]:
    if which == "gpu":
        files = glob.glob(os.path.join(HERE, "*.cu")) + glob.glob(os.path.join(HERE, "*.cuh")) + \
            [os.path.join(HERE, "..", "..", "include", "vulcan_b200.h")]
    elif which == "core":
        files = [os.path.join(HERE, "vulcan_core.cpp")]
    else:
        raise SystemExit(f"unknown library {which}")
    return sorted(files, key=os.path.basename)


def digest(which: str) -> str:
    h = hashlib.sha256()
    for f in sources(which):
        h.update(os.path.basename(f).encode())
        with open(f, "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()


if __name__ == "__main__":
    print(digest(sys.argv[1]))
