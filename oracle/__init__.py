"""ORACLE -- test infrastructure only: the float64 CPU restatement of the
reference's per-step loop (vlasov_oracle.cpp, oracle.py) and the pure-Python
ran2 (ran2.py).  Never imported by the product path."""
