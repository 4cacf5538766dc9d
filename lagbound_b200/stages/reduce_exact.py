#!/usr/bin/env python3
"""Drop-in for the exact-reduction stage (src/lagbound/_core/reduce_exact.py) on a B200:
    reduce_exact.py <tag> [label files ...]
reads data/<tag>/{graph.json, keys.npy} under the working directory, writes data/<tag>__rx/ (graph.json, keys.npy,
weights.npy, vol.npy, meta.json, group_of.npy and the restricted label files) and prints the same lines."""
import os
import sys

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))


def main(argv=None):
    from lagbound_b200 import reduce as R
    R.main(sys.argv[1:] if argv is None else argv)


if __name__ == "__main__":
    main()
