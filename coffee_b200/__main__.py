"""``python -m coffee_b200 <driver> -c config.toml``: see coffee_b200.cli."""
import sys

from .cli import main

sys.exit(main())
