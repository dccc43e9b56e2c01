"""ORACLE — test infrastructure only (tests/, __graft_entry__.smoke(), bench.py's CPU baseline).

CPU restatements of tgautam03/xAdvCool's solver path used to check the CUDA product. Nothing in the
product package imports this.
"""
