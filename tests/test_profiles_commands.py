"""The commands the ncu summaries under profiles/ give still run committed files (CPU).

Every `python <script> ...` command quoted in one of those summaries must name a script of this
repository, and every `--option` it passes must be one that script defines, so that a reader can
re-run the command that made the figures.
"""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PROFILES = os.path.join(ROOT, "profiles")
CMD = re.compile(r"python[ \t]+([\w./-]+\.py)((?:[ \t]+-[^\s`]+(?:[ \t]+[^\s`-][^\s`]*)?)*)")


def _commands():
    out = []
    for name in sorted(os.listdir(PROFILES)):
        if name.endswith(".md"):
            with open(os.path.join(PROFILES, name)) as f:
                for m in CMD.finditer(f.read()):
                    out.append((name, m.group(1), m.group(2)))
    return out


def test_profiles_quote_commands():
    assert len(_commands()) >= 5


@pytest.mark.parametrize("name,script,args", _commands())
def test_profile_command_runs_committed_files(name, script, args):
    path = os.path.join(ROOT, script)
    assert os.path.isfile(path), f"{name}: {script} is not a file of the repository"
    with open(path) as f:
        src = f.read()
    for opt in re.findall(r"(?<!\S)(--[\w-]+)", args):
        assert f'"{opt}"' in src, f"{name}: {script} defines no option {opt}"
    for wl in re.findall(r"--workload\s+(\S+)", args):
        assert f'"{wl}"' in src, f"{name}: {script} has no workload {wl}"
