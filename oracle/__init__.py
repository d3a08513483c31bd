"""CPU oracle package: TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU
baseline / reference legs may import this package, and only as the checker
or the timed CPU baseline.  The product (``gb_kun_b200``) never imports it.
"""
