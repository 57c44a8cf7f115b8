// placeholder, filled in by the HDF5 reader/writer
