#!/bin/sh
# Regenerate tests/golden/ckpt2d_ref_n2.bin.gz: a 2D checkpoint written by the
# reference's own cell_gh200 (oracle/_ref, built by `make -C oracle ref`), 2
# cells of radius 12 on a 301^2 lattice after 3 steps. Needs a GPU.
set -e
here=$(cd "$(dirname "$0")" && pwd)
out=${1:-$here}
tmp=$(mktemp -d)
"$here/../../oracle/_ref/cell_gh200" --N 2 --radius 12 --rho 0.01 --seed 3 --t-end 0.03 \
    --checkpoint-dir "$tmp" > "$tmp/log.txt"
gzip -9 -n -c "$tmp/checkpoint.bin" > "$out/ckpt2d_ref_n2.bin.gz"
rm -rf "$tmp"
