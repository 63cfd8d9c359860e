#!/bin/sh
# Regenerate tests/golden/ckpt3d_ref_n2.pf3d.gz: a PF3D checkpoint written by
# the reference's own cell_gh200_3d (oracle/_ref, built by `make -C oracle
# ref`), 2 periodic cells of radius 4 (lambda 3, 32^3 bricks) on a 48^3
# lattice after 3 steps. Needs a GPU.
set -e
here=$(cd "$(dirname "$0")" && pwd)
out=${1:-$here}
tmp=$(mktemp -d)
"$here/../../oracle/_ref/cell_gh200_3d" --N 2 --radius 4 --lambda 3 --rho 0.005 --seed 3 \
    --t-end 0.03 --print-interval 0 --checkpoint-dir "$tmp" > "$tmp/log.txt"
gzip -9 -n -c "$tmp/checkpoint.pf3d" > "$out/ckpt3d_ref_n2.pf3d.gz"
rm -rf "$tmp"
