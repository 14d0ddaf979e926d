# tests/golden/validation_results.json was written on one B200 by
cd ls-sph-benchmarks_b200 && python -m lssph.validation --out ../tests/golden/validation_results.json
# (the same runs as: python bench.py --validate).  Deviation from the Ghia et al. (1982) table,
# read in place from the reference checkout:
cd ls-sph-benchmarks_b200 && python -m lssph.validation --compare ../tests/golden/validation_results.json \
    --ghia "$LSSPH_REFERENCE_ROOT/analysis/benchmarks/Ghia_1982_Re_1000.csv"
