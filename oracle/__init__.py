"""Oracle: CPU restatements of the reference's depth-LUT physics and separable
dose engine, used ONLY as the checker in ``tests/``, in ``__graft_entry__.smoke()``
and as the CPU baseline in ``bench.py``.  The product package never imports it.
"""
