"""python -m inchman_b200 [--output FILE] [--p NAME=VALUE]... model.xml (see cli.py)."""
import sys

from .cli import main

sys.exit(main())
