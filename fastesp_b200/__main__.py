"""``python -m fastesp_b200 esp|build-native|selftest`` (see fastesp_b200.cli)."""
import sys

from .cli import main

sys.exit(main())
