"""``python -m rigidfibers_kth_b200 PARAMETERS LAYOUT``: see cli.py."""
import sys

from .cli import main

sys.exit(main())
