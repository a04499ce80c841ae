"""The roofline probes measure what they claim.

* ctas_probe_smem_gather: conflict-free 32-bit shared loads. It cannot exceed
  the shared-memory pipe's 128 B per clock per SM at the highest SM clock
  (2.1 GHz bounds every B200 clock), and a probe that the compiler did not
  shorten lands well above half of it.
* ctas_probe_l2_read: 16-byte reads of an L2-resident buffer. They lie above the
  DRAM copy bandwidth (the buffer does not leave L2) and below the
  shared-memory figure.
"""
import pytest

from ctas_b200 import ct

pytestmark = pytest.mark.gpu


def _sms():
    import torch
    return torch.cuda.get_device_properties(0).multi_processor_count


def test_smem_probe_within_the_pipe():
    got = ct.probe_smem_gather(0)
    cap = 128.0 * _sms() * 2.1e9
    assert 0.5 * cap < got <= cap, (got, cap)


def test_l2_probe_between_dram_and_smem():
    l2 = ct.probe_l2_read(0)
    smem = ct.probe_smem_gather(0)
    assert 2e12 < l2 < smem, (l2, smem)
