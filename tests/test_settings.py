"""CPU: derived settings follow src/swspectrometer.cpp:166-231."""
from swspec_b200.settings import from_ini_values


def test_c1_buffer_plan_default_32mb():
    s = from_ini_values(fft_points=32768, fft_integ_seconds=1.0, fft_overlap_factor=1,
                        BandwidthHz=16e6, bits_per_sample=2, source_channels=16)
    assert s.averaged_ffts == 976          # int(fs*T/N), not 977
    assert s.raw_fullfft_bytes == 131072
    assert s.max_buffers_per_spectrum == 61 and s.max_specffts_per_buffer == 16
    assert s.core_overlapped_ffts == 16 and s.rawbuf_size == 2 * 1024 * 1024


def test_c3_buffer_plan():
    s = from_ini_values(fft_points=65536, fft_integ_seconds=1.0, fft_overlap_factor=1,
                        BandwidthHz=32e6, bits_per_sample=2, source_channels=16)
    assert s.averaged_ffts == 976 and s.raw_fullfft_bytes == 262144
    assert s.max_buffers_per_spectrum == 61 and s.core_overlapped_ffts == 16
    assert s.rawbuf_size == 4 * 1024 * 1024


def test_overlap_core_ffts_and_packed_spectra():
    s = from_ini_values(fft_points=4096, fft_integ_seconds=0.01, fft_overlap_factor=2,
                        BandwidthHz=8e6, bits_per_sample=2, source_channels=4)
    # 16e6*0.01/4096 = 39 FFTs, 4096 B each -> fits; several spectra per buffer
    assert s.averaged_ffts == 39 and s.max_spectra_per_buffer >= 1
    assert s.core_overlapped_ffts == 2 * 39 - 1


def test_pcal_derivation_and_disable():
    s = from_ini_values(fft_points=3200000, fft_integ_seconds=10.0, BandwidthHz=16e6,
                        bits_per_sample=2, source_channels=16, extract_PCal=True)
    assert s.pcal_tonebins == 32 and s.pcal_rotatorlen == 3200 and s.pcal_pulses_per_fft == 1000
    s2 = from_ini_values(fft_points=32768, BandwidthHz=16e6, extract_PCal=True)
    assert not s2.extract_PCal            # 32768 % 3200 != 0 disables PCal
