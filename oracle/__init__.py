"""CPU checkers (test infrastructure only): the restatement of the reference's
hot path and, where the reference tree is present, the unchanged reference
built from its sources.  SNC_REF names that tree (default /root/reference)."""
import os

REF_ROOT = os.environ.get("SNC_REF", "/root/reference")
