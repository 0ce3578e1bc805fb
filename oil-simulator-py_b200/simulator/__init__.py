"""Drop-in for the reference's ``simulator`` package (src/simulator/)."""
