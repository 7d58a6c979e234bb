"""The classifier shipped with the package (heimdall_multibeam_b200/
classifier_survey.npy, trained by heimdall_multibeam_b200.training on 10^5
candidates of survey-shaped gulps: 1024 channels, 64 us, 2^18 samples, DM
0-2000) on held-out survey-shaped gulps it has not seen: scored through
hd_score_candidates (patches extracted and scored on the GPU after the
merge), at its stored threshold it keeps >= 99 % of the plain list's recall
of injected S/N >= 8 pulses and removes >= 90 % of the RFI candidates.  The
plain candidate list is the pipeline's own (cleaning off, so that the RFI
reaches it) and stays unchanged."""
import json
import os

import numpy as np
import pytest

import heimdall_multibeam_b200 as H
from heimdall_multibeam_b200 import training

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

HERE = os.path.dirname(os.path.abspath(H.__file__))


def test_shipped_classifier_on_held_out_survey_gulps(hdb):
    params = np.load(os.path.join(HERE, "classifier_survey.npy"))
    with open(os.path.join(HERE, "classifier_survey.json")) as f:
        meta = json.load(f)
    assert params.shape == (int(H.lib().hd_classifier_param_count()),)
    thresh = meta["threshold"]
    with H.Classifier(seed=0) as clf:
        clf.set_params(params)
        d = training.collect(H, torch, range(300000, 300032), classifier=clf, patches=False)
    assert len(d["score"]) == len(d["label"]) > 1000
    r = training.recall_and_reduction(d, d["score"], thresh)
    print(json.dumps(r))
    assert r["pulses"] > 800 and r["rfi_candidates"] > 1000
    assert r["recall_classified"] >= 0.99 * r["recall_plain"]
    assert r["rfi_kept"] <= 0.1
