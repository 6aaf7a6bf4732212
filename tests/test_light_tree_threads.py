"""The host light-tree builder on several threads (tpt_light_tree_build_threads).

Subtrees of 1,024 or more emitters go to other threads; node numbering is
fixed by the subtree sizes, so the tree must not depend on the thread count.
The SHA-256 prefixes below are of the node arrays the one-thread builder wrote
for these seeded scenes (the 10,000-emitter grid scene, a 3,000-emitter one,
the lit Cornell box, the 64-patch box); every thread count must give them.
"""
import hashlib

import pytest

import tpt
import tpt_scenes

CASES = {
    "grid_10k": (lambda: tpt_scenes.grid_scene(), "df70b8c5965d29dc90a0e92047702336", 19999),
    "grid_3k": (lambda: tpt_scenes.grid_scene(seed=7, n_side=8, n_emissive_tris=3000),
                "ad11868a9f7b160534a4716fbc96ede8", 5999),
    "cornell_lights": (lambda: tpt_scenes.cornell_lights(3, tpt_scenes.OPENPBR), "ca6e53718da7f68e4b17ebf9b539d3fa", 7),
    "patches": (lambda: tpt_scenes.cornell_patches(), "4f0893359a3814c82c4c318fb257bb57", 3),
}


@pytest.mark.parametrize("name", list(CASES))
def test_tree_independent_of_threads(name):
    make, digest, n_nodes = CASES[name]
    sc = make()
    for threads in (1, 2, 3, 16, 0):
        nodes, root = tpt.build_light_tree(sc, threads=threads)
        assert root == 0 and len(nodes) == n_nodes
        assert hashlib.sha256(nodes.tobytes()).hexdigest()[:32] == digest, threads
