"""Writes the reference's demo scenes 1..7 (beatbox.reference_scenes) as the data files of this
folder: scene_<k>.npz in the beatbox.io scene format.

  python beat-box_b200/beatbox/scene_data/make_scene_data.py
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from beatbox import io  # noqa: E402
from beatbox.reference_scenes import SCENES  # noqa: E402


def main():
    for k, make in SCENES.items():
        sc = make()
        io.save_scene(sc, os.path.join(HERE, f"scene_{k}.npz"))
        print(f"scene_{k}: {sc['n']} bodies")


if __name__ == "__main__":
    main()
