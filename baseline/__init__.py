"""The reference's own GPU sweep, built for sm_100a from its sources (`ref_gpu`)."""
