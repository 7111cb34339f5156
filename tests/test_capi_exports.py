"""The C-ABI library loads and exports every entry point its headers declare."""
import glob
import os
import re

from conftest import ROOT


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        names |= set(re.findall(r"\b(svo_\w+)\s*\(", text))
    return names


def test_exports(svo_mod):
    names = _declared()
    assert len(names) >= 25
    L = svo_mod.lib()
    missing = [n for n in sorted(names) if not hasattr(L, n)]
    assert not missing, missing


def test_cli_built(svo_mod):
    assert os.access(svo_mod.CLI_PATH, os.X_OK)
