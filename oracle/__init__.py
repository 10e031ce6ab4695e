"""CPU oracle for the Tier-3 step -- TEST INFRASTRUCTURE ONLY.

A numpy restatement of the reference's algorithm (src/model_outdoor/
spread_3d.py and physics_3d/), each function citing the reference lines it
follows.  It is pinned against the reference's committed golden vectors and
against states captured from the reference solver itself
(tests/golden/*.npz), and it is used only as the checker in tests/, in
``__graft_entry__.smoke()`` and as the timed CPU baseline in ``bench.py``.
The product path (firewebapp_b200) never imports it.
"""
