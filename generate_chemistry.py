#!/usr/bin/env python
"""Generator CLI (see chemgen_b200/cli.py): --mode getrates --language cuda."""
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

from chemgen_b200.cli import main

if __name__ == "__main__":
    sys.exit(main())
