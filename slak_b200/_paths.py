"""Locations of the in-tree shared libraries built by ``slak_b200.build``."""
import os

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO_DIR = os.path.dirname(PKG_DIR)
LIB_DIR = os.path.join(PKG_DIR, "lib")

LIB_SLAK = os.path.join(LIB_DIR, "libslak_b200.so")          # CUDA product library (C-ABI)
LIB_MESHGEN = os.path.join(LIB_DIR, "libslak_meshgen.so")     # host mesh generators
LIB_ORACLE = os.path.join(REPO_DIR, "oracle", "_build", "libslak_oracle.so")
LIB_REF = os.path.join(REPO_DIR, "oracle", "_ref", "libslak_ref.so")
DROPIN_MAIN = os.path.join(REPO_DIR, "oracle", "_ref", "slak_main_dropin")   # the reference's main.cpp, our library
DEMO_BIN = os.path.join(LIB_DIR, "slak_demo")
INCLUDE_DIR = os.path.join(REPO_DIR, "include")
CSRC_DIR = os.path.join(PKG_DIR, "csrc")
