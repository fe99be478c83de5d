#!/usr/bin/env bash
# Install the unmodified reference (THUHoloLab/PtychoX, its python/ package) into baseline/_ref
# for bench.py's reference arm and the drop-in tests.  Run in the build container, where the
# reference checkout exists; baseline/_ref is git-ignored and travels with the repository to
# the GPU machine.
#
#   baseline/install_reference.sh [REFERENCE_CHECKOUT]
#
# The reference's setup.py builds its three pybind11/cuFFT extensions (ptychoX.{base,fpm,coded}._C)
# and writes build files next to its sources, so the package is copied to a scratch directory
# first.  TORCH_CUDA_ARCH_LIST=10.0a compiles the extensions for B200 (sm_100a); the reference's
# own default is 8.6.  The driver scripts (train_*.py) are copied beside the package: the
# coded driver holds fd_loss (train_coded.py:101-107), which the reference arm imports.
set -euo pipefail
SRC="${1:?usage: $0 REFERENCE_CHECKOUT (the PtychoX repository root)}"
HERE="$(cd "$(dirname "$0")" && pwd)"
DEST="$HERE/_ref"
TMP="$(mktemp -d)"
trap 'rm -rf "$TMP"' EXIT
cp -r "$SRC/python" "$TMP/src"
chmod -R u+w "$TMP/src"
find "$TMP/src" -name '__pycache__' -prune -exec rm -rf {} +
rm -rf "$TMP/src/build" "$TMP/src/.torch_extensions"
rm -rf "$DEST"
TORCH_CUDA_ARCH_LIST="10.0a" MAX_JOBS="${MAX_JOBS:-8}" \
  python -m pip install --no-index --no-build-isolation --find-links /opt/wheelhouse \
  --target "$DEST" "$TMP/src"
cp "$TMP/src"/train_ptychography.py "$TMP/src"/train_fpm.py "$TMP/src"/train_coded.py "$DEST"/
echo "reference installed in $DEST"
