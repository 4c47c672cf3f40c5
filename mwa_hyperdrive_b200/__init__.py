"""B200-native sky-model predictor, DI calibration and peeling for MWA data,
behind mwa_hyperdrive's SkyModeller / calibrate / peel interfaces."""

__version__ = "0.1.0"
