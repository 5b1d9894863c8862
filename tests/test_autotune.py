"""The autotuner's host logic (no GPU): merging the tuning runs of the two
chain-order builds, and the tables the build bakes from the result."""
import json
import os

from intception_b200 import autotune
from intception_b200.emit import eri_emitter


def _run(order, ms_by_tag):
    classes = {}
    for tag, (fp64, fp32) in ms_by_tag.items():
        classes[tag] = {'minb': [0, 1, 2, 3] if order == 'level' else [3, 2, 1, 0],
                        'ms': {'fp64_cart': [fp64, fp64 + 1], 'fp64_sph': [fp64 + 0.5, fp64],
                               'fp32_cart': [fp32, fp32 + 1], 'fp32_sph': [fp32 + 1, fp32]}}
    return {'meta': {'chain_order': order}, 'classes': classes}


def test_merge_picks_the_faster_order_and_fp32(tmp_path):
    a = tmp_path / 'dfs.json'
    b = tmp_path / 'level.json'
    a.write_text(json.dumps(_run('dfs', {'2221': (10.0, 7.0), '1000': (1.0, 1.5)})))
    b.write_text(json.dumps(_run('level', {'2221': (9.0, 6.5), '1000': (1.2, 1.6)})))
    out = tmp_path / 'tuning.json'
    merged = autotune.merge([str(a), str(b)], str(out))
    assert merged['2221']['order'] == 'level' and merged['2221']['minb'] == [0, 1, 2, 3]
    assert merged['1000']['order'] == 'dfs' and merged['1000']['minb'] == [3, 2, 1, 0]
    assert merged['2221']['fp32'] is True   # FP32 kernel at least 3 % faster in both outputs
    assert merged['1000']['fp32'] is False  # slower: the FP32 tier leaves this class in FP64
    assert json.loads(out.read_text())['classes'] == merged


def test_committed_tuning_covers_every_tuned_class():
    path = os.path.join(os.path.dirname(autotune.__file__), 'tuning.json')
    with open(path) as fh:
        tun = json.load(fh)['classes']
    tags = {'%d%d%d%d' % c for c in eri_emitter.canonical_classes(2)}
    # and the emitted f classes in canonical order (autotune --classes f)
    tags |= {'%d%d%d%d' % c for c, _ in eri_emitter.emitted_classes()
             if max(c) == 3 and c[0] >= c[1] and c[2] >= c[3]}
    assert tags == set(tun)
    for ent in tun.values():
        assert len(ent['minb']) == 4 and all(0 <= m < len(autotune.MINB_VALUES) for m in ent['minb'])
        assert ent['order'] in ('dfs', 'level') and isinstance(ent['fp32'], bool)
