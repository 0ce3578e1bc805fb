"""Drop-in for the reference's ``solver`` package (src/solver/)."""
