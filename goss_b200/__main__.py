"""``python -m goss_b200 <command>``: see :mod:`goss_b200.cli`."""
from .cli import app

if __name__ == "__main__":
    app(prog_name="goss_b200")
