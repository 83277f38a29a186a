"""CPU oracle for the CKKS evaluation core.

TEST INFRASTRUCTURE ONLY.  Nothing in the product (``cipher-pu_b200/``) imports
this package.  Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s
``cpu_baseline`` leg / ``--impl reference`` arm may import or run it, and only as
the checker or as the timed CPU baseline, never as the thing measured or shipped.

What it holds: a numpy / Python-int restatement of the reference's hot-path
algorithms (YI-HAIBO/cipher-pu), each function citing the reference file:line it
follows, plus CPU restatements of the RNS-CKKS pieces the reference does not
have (hybrid keyswitch with ModUp/ModDown, RNS rescale, CRT, DARE over RNS),
written from the CKKS mathematics.

Parity pinning: ``tests/test_oracle_pins.py`` checks this oracle against
golden vectors generated by importing the reference's own Python functions
(``tests/golden/make_golden.py``), against the reference's committed twiddle
and modulus-chain fixtures, and against its known-answer constants.  The RNS
hybrid keyswitch / RNS rescale / DARE-over-RNS parts have no reference code;
they are pinned by an independent big-integer restatement of the whole
ct-mult (``oracle.rns_ckks.bigint_ct_mul``: CRT-composed integers, schoolbook
negacyclic products, exact division by the special prime and by q_t).
"""
