"""The scene inputs behind the image fixtures are what the fixtures were made from: the
scene generators must still produce them bit for bit (tests/golden/scene_digests.json,
written by tests/golden/make_golden.py digests).  A change to a generator that fails this
needs the affected fixtures made again from the reference."""
import json
from pathlib import Path

import pytest

from golden.make_golden import image_fixture_scenes, scene_digest

DIGESTS = json.loads((Path(__file__).resolve().parent / "golden" / "scene_digests.json").read_text())


@pytest.mark.parametrize("name,builder", image_fixture_scenes(), ids=[n for n, _ in image_fixture_scenes()])
def test_fixture_scene_inputs_unchanged(name, builder):
    assert scene_digest(builder()) == DIGESTS[name]
