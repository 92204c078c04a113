"""Host build of the reference's own sources (test infrastructure)."""
from __future__ import annotations

import os
from pathlib import Path


def reference_root() -> Path | None:
    """The reference source tree: $SMAUG_REFERENCE, else a `reference`
    directory beside this repository; None when neither holds dev/smaug/src
    (a machine without the reference sources uses the prebuilt files)."""
    repo = Path(__file__).resolve().parents[2]
    for cand in (os.environ.get("SMAUG_REFERENCE"), repo.parent / "reference"):
        if cand and (Path(cand) / "dev" / "smaug" / "src").is_dir():
            return Path(cand)
    return None
