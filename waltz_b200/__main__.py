"""`python -m waltz_b200`: the command-line codec (waltz_b200.cli)."""
import sys

from .cli import main

sys.exit(main())
