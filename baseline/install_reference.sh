#!/bin/sh
# Install the reference package (quantem, pure Python) into baseline/_ref, where
# `bench.py --impl reference --torch-gpu` imports it to time the reference's own
# PyTorch iteration on the GPU.  baseline/_ref is git-ignored and travels with
# the working tree.  pip needs the package's build backend (hatchling); when the
# offline wheelhouse lacks it, the package tree the wheel would install
# (src/quantem) is copied instead.
#
#   sh baseline/install_reference.sh <reference checkout>
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
SRC=${1:?usage: install_reference.sh <reference checkout>}
TMP=$(mktemp -d)
cp -r "$SRC" "$TMP/src"
if python -m pip install --no-index --no-build-isolation --no-deps --find-links /opt/wheelhouse \
    --target "$HERE/_ref" "$TMP/src" >/dev/null 2>&1; then
  echo "installed with pip into $HERE/_ref"
else
  mkdir -p "$HERE/_ref"
  rm -rf "$HERE/_ref/quantem"
  cp -r "$TMP/src/src/quantem" "$HERE/_ref/quantem"
  echo "pip could not build the package (build backend missing); copied the package tree into $HERE/_ref"
fi
rm -rf "$TMP"
