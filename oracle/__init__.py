"""CPU oracle of the extended-KKS step: TEST INFRASTRUCTURE ONLY.

Imported by the test-suite, by ``__graft_entry__.smoke()`` (as the checker) and
by the CPU-baseline leg of ``bench.py``; never by the product package.
"""
