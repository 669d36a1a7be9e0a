// Instantiations the oracle's ingest binding uses (16-bit detector files).
template class ImageTiff<unsigned short>;
template class ImageCalibration<unsigned short>;
