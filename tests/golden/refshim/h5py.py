"""Empty stand-in: the reference imports h5py only for Monitor.save to HDF5."""
