#!/bin/sh
# Copies the reference's own test data (kikuchipy's nickel scan as h5ebsd, the nickel and GaN
# masters, kikuchipy's refined orientations of the scan; CC BY 4.0, see the reference's
# testdata/nickel/LICENSE) into tests/data/, which git ignores: the tests that need these files
# find them there (or under $ZEBSDSOLVE_TESTDATA) and skip when they are absent.
#
#   tests/golden/copy_testdata.sh <the reference's testdata directory>
#   ZEBSDSOLVE_REFERENCE=<the reference checkout> tests/golden/copy_testdata.sh
set -e
SRC=${1:-${ZEBSDSOLVE_REFERENCE:+$ZEBSDSOLVE_REFERENCE/testdata}}
if [ -z "$SRC" ]; then
  echo "usage: $0 <reference testdata directory> (or set ZEBSDSOLVE_REFERENCE to the reference checkout)" >&2
  exit 2
fi
DST=$(dirname "$0")/../data
mkdir -p "$DST/nickel" "$DST/gan"
for f in patterns_v2.h5 Ni_master_20kV.npz reference_quaternions.f32 LICENSE; do
  cp "$SRC/nickel/$f" "$DST/nickel/$f"
done
cp "$SRC/gan/GaN_master_20kV.npz" "$DST/gan/GaN_master_20kV.npz"
