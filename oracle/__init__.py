"""TEST INFRASTRUCTURE ONLY: CPU oracles for the PR flash (see oracle/oracle.py).

``REF_ROOT`` is where the reference's sources are read from when the
compiled-reference oracle is built (oracle/Makefile's ``REF``): the
``OCP_REFERENCE`` environment variable, else the default below."""
import os

REF_ROOT = os.environ.get("OCP_REFERENCE", "/root/reference")
